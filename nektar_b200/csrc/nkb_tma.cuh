// Bulk (TMA) copies into shared memory completed through an mbarrier, for
// sm_100a. Untiled cp.async.bulk from this GPU's own global memory into the
// issuing CTA's shared memory; no cluster multicast anywhere.
//
// Rules kept by the callers: source and destination 16-byte aligned, size a
// multiple of 16 bytes. Every wait is bounded: after kMaxPolls failed polls
// the waiter records an error word, keeps waiting for at most the same
// bound again so no copy is left writing into shared memory of a CTA that
// has exited, and then returns false.
#pragma once

#include <cstdint>

namespace nkb
{

constexpr unsigned kMaxPolls = 1u << 24; // try_wait polls (each may suspend briefly)

__device__ __forceinline__ uint32_t SmemAddr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void MbarInit(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count)
                 : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void MbarInval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

__device__ __forceinline__ void MbarArriveExpectTx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)),
                 "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy, completion counted on bar (bytes % 16 == 0)
__device__ __forceinline__ void BulkG2S(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                 "%2, [%3];" ::"r"(SmemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                 : "memory");
}

// bulk prefetch of [src, src+bytes) into L2 (bytes % 16 == 0, src 16-byte
// aligned); no shared memory, no completion to wait for
__device__ __forceinline__ void BulkPrefetchL2(const void *src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool MbarTryWait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(SmemAddr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// first bound of a kernel's bounded waits: word [1] of its error buffer
// holds bound + 1 when a test has set one (nkb_op_set_wait_limit; 1: give up
// at once), 0 for the default kMaxPolls
__device__ __forceinline__ unsigned WaitPolls(const int *err)
{
    const unsigned v = err ? static_cast<unsigned>(__ldg(err + 1)) : 0u;
    return v ? v - 1u : kMaxPolls;
}

// Bounded wait for phase `parity` of bar. Returns true when the phase
// completed within `polls` polls; otherwise *err is set and the wait goes on
// for at most kMaxPolls more polls (so a copy still in flight lands before
// the CTA can exit) and returns false. `polls` is kMaxPolls unless a test
// lowers it (WaitPolls) to make the first bound run out.
__device__ __forceinline__ bool MbarWaitBounded(uint64_t *bar, uint32_t parity, int *err, int code,
                                                unsigned polls = kMaxPolls)
{
    for (unsigned n = 0; n < polls; ++n)
        if (MbarTryWait(bar, parity))
            return true;
    if (err)
        atomicExch(err, code);
    for (unsigned n = 0; n < kMaxPolls; ++n)
        if (MbarTryWait(bar, parity))
            return false;
    return false;
}

} // namespace nkb
