// Test infrastructure only (oracle). A minimal stand-in for
// boost::alignment::aligned_allocator so that the reference's tinysimd
// headers (LibUtilities/SimdLib/allocator.hpp) compile without Boost.
// Only the members std::vector needs are provided.
#ifndef NKB_ORACLE_SHIM_ALIGNED_ALLOCATOR_HPP
#define NKB_ORACLE_SHIM_ALIGNED_ALLOCATOR_HPP

#include <cstddef>
#include <new>

namespace boost
{
namespace alignment
{

template <class T, std::size_t Align> class aligned_allocator
{
public:
    using value_type = T;
    template <class U> struct rebind
    {
        using other = aligned_allocator<U, Align>;
    };

    aligned_allocator() noexcept = default;
    template <class U>
    aligned_allocator(const aligned_allocator<U, Align> &) noexcept
    {
    }

    T *allocate(std::size_t n)
    {
        std::size_t a = Align < alignof(T) ? alignof(T) : Align;
        return static_cast<T *>(::operator new(n * sizeof(T), std::align_val_t(a)));
    }
    void deallocate(T *p, std::size_t) noexcept
    {
        std::size_t a = Align < alignof(T) ? alignof(T) : Align;
        ::operator delete(p, std::align_val_t(a));
    }
    template <class U> bool operator==(const aligned_allocator<U, Align> &) const noexcept
    {
        return true;
    }
    template <class U> bool operator!=(const aligned_allocator<U, Align> &) const noexcept
    {
        return false;
    }
};

} // namespace alignment
} // namespace boost

#endif
