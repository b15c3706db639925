// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a:
// tensor-memory allocation, shared-memory matrix descriptors, TF32 MMAs with
// FP32 accumulation in tensor memory, commit to an mbarrier, tensor-memory
// loads and the fences that order them.
//
// Operand layout (K-major, no swizzle; byte offsets within one 128-row
// operand of one 8-wide K step, 4096 bytes):
//   element (m, k): (m / 8) * 256 + (k / 4) * 128 + (m % 8) * 16 + (k % 4) * 4
//   descriptor: leading-byte offset 128 (K chunk), stride-byte offset 256
//   (8-row group)
// A B operand (N rows, K-major) uses the same form with N in place of M.
// Only K-major operands are used: with the MN-major bit set, TF32 MMAs on
// sm_100a produced zeros for every no-swizzle layout and stride assignment
// tried.
//
// Precision: a TF32 MMA reads the top 19 bits of each FP32 operand. An FP32
// value a is split into a_hi = tf32(a) (round to nearest) and a_lo = a - a_hi
// (exact); constant tables are split the same way from their FP64 values.
// With B = [b_hi | b_lo] side by side in N, the two MMAs a_hi x B and a_lo x B
// accumulated into one tensor-memory tile hold a_hi b_hi + a_lo b_hi in the
// first half of the columns and a_hi b_lo + a_lo b_lo in the second; their
// sum is a b to about 2^-21 relative (the truncation of a_lo and b_lo), an
// FP32-class product (Markidis et al., IPDPSW 2018, splitting operands into
// high and low parts for tensor cores).
#pragma once

#include <cstdint>

namespace nkb
{
namespace tc
{

constexpr uint32_t kOperandBytes = 4096; // one 128 x 8 TF32 operand step

__device__ __forceinline__ uint32_t SmemU32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor (no swizzle, base offset 0, version 1)
__device__ __forceinline__ uint64_t Desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ uint64_t DescKMajor(uint32_t saddr)
{
    return Desc(saddr, 128, 256);
}

// instruction descriptor: TF32 x TF32 -> FP32, M = 128, A and B K-major
__host__ __device__ constexpr uint32_t IDescTf32(int n)
{
    return (1u << 4)                    // accumulator FP32
           | (2u << 7) | (2u << 10)     // A, B TF32
           | (uint32_t(n >> 3) << 17)   // N / 8
           | (uint32_t(128 >> 4) << 24); // M / 16
}

// D[tmem] (+)= A[adesc] x B[bdesc], issued by one thread
__device__ __forceinline__ void MmaTf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, bool accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                 :
                 : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1 : 0)
                 : "memory");
}

// the mbarrier gets one arrival when every MMA this thread issued before has
// completed
__device__ __forceinline__ void Commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     SmemU32(bar))
                 : "memory");
}

// tensor-memory allocation by one whole warp; the base address goes to *slot
__device__ __forceinline__ void Alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemU32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void Dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void FenceBeforeSync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void FenceAfterSync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// generic-proxy shared-memory writes become visible to the tensor cores
__device__ __forceinline__ void FenceProxyAsync()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane (the warp
// reads its quarter of the lanes; taddr carries the warp's lane base)
__device__ __forceinline__ void Ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
                 "%10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int c = 0; c < 16; ++c)
        v[c] = __uint_as_float(r[c]);
}

__device__ __forceinline__ void WaitLd()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float Tf32Hi(float a)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
    return __uint_as_float(r);
}

// A K-major operand of 128 rows: 8-row groups SBO bytes apart, the two
// 4-wide K chunks of a group LBO bytes apart (LBO >= 128, SBO >= LBO + 128),
// one 8-wide K step STEP bytes. The standard packing (256, 128) is dense; the
// padded one (272, 144) shifts consecutive row groups by 4 banks and the
// second K chunk by 4 more, which makes the scalar column stores of a warp
// (8 row groups, or 4 groups x 8 K values) hit distinct banks, for 1/16 more
// shared memory.
template <int SBO_, int LBO_> struct ALayout
{
    static constexpr int SBO = SBO_, LBO = LBO_, STEP = 16 * SBO_;
    static_assert(LBO_ >= 128 && SBO_ >= LBO_ + 128 && SBO_ % 16 == 0 && LBO_ % 16 == 0,
                  "K-major operand strides");
    __host__ __device__ static constexpr uint32_t Off(int m, int k)
    {
        return uint32_t(k >> 3) * uint32_t(STEP) + uint32_t(m >> 3) * uint32_t(SBO) +
               uint32_t((k & 7) >> 2) * uint32_t(LBO) + uint32_t(m & 7) * 16u + uint32_t(k & 3) * 4u;
    }
};
using ALayoutStd = ALayout<256, 128>;
using ALayoutPad = ALayout<272, 144>;

// byte offsets of element (m, k) in a standard operand of 8-wide K steps
__host__ __device__ constexpr uint32_t OffK(int m, int k)
{
    return ALayoutStd::Off(m, k);
}

// B operand (K-major, nrows rows padded to 8): element (n, k); one K step
// holds nrows * 32 bytes
__host__ __device__ constexpr uint32_t OffB(int n, int k, int nrows)
{
    return uint32_t(k >> 3) * uint32_t(nrows) * 32u + uint32_t(n >> 3) * 256u +
           uint32_t((k & 7) >> 2) * 128u + uint32_t(n & 7) * 16u + uint32_t(k & 3) * 4u;
}

} // namespace tc
} // namespace nkb
