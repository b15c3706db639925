// Self-test of the tcgen05 building blocks used by the tensor-core Hex kernel
// (nkb_hex_tc.cuh): one 128-row tile D = A B with A written by the kernel's
// row writer or its column writer (split into TF32 high and low parts), B
// in the K-major table form, the MMA pair issued and committed to an
// mbarrier, and the raw tensor-memory columns read back. A test compares D
// with A B computed on the host; it pins the layout conventions the kernel
// relies on.
#include "nkb_hex_kernel.cuh"
#include "nkb_internal.h"
#include "nkb_tma.cuh"

#include <cuda_runtime.h>

#include <vector>

namespace nkb
{
namespace
{
constexpr int kSelfMaxK = 16, kSelfMaxN = 64;

// one CTA of 128 threads; thread t owns row t. A: 128 x K row-major, B: K x
// N row-major (global); D: 128 x N; info: [0] tensor-memory base, [1] 1 if
// the MMA wait completed
__global__ void __launch_bounds__(128, 1)
    k_tc_selftest(int colw, int n, int ks, const float *__restrict__ A, const float *__restrict__ B,
                  float *__restrict__ D, unsigned *info, int *err)
{
    __shared__ __align__(1024) unsigned char sa[2 * 2 * tc::ALayoutPad::STEP];
    __shared__ __align__(1024) unsigned char sb[kSelfMaxN * kSelfMaxK * 4];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    const int t = threadIdx.x, warp = t >> 5, K = 8 * ks;
    // high part: two K steps; low part after them (either layout fits)
    const int step    = colw == 2 ? tc::ALayoutPad::STEP : tc::ALayoutStd::STEP;
    unsigned char *hi = sa, *lo = sa + 2 * step;
    for (int o = t * 16; o < int(sizeof(sa)); o += 128 * 16)
        *reinterpret_cast<float4 *>(sa + o) = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int o = t * 16; o < int(sizeof(sb)); o += 128 * 16)
        *reinterpret_cast<float4 *>(sb + o) = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    // B: element (row n, k) of the K-major table holds B[k][n]
    for (int e = t; e < n * K; e += 128)
    {
        const int r = e / K, k = e % K;
        *reinterpret_cast<float *>(sb + tc::OffB(r, k, n)) = B[k * n + r];
    }
    // A: the kernel's writers. Rows: this thread's row; columns: thread t < K
    // writes column t over all 128 rows, 8 rows at a time, rotated by t
    if (!colw)
    {
        float v[kSelfMaxK];
#pragma unroll
        for (int k = 0; k < kSelfMaxK; ++k)
            v[k] = k < K ? A[t * K + k] : 0.f;
        if (ks == 1)
            tcd::WriteRowK<tc::ALayoutStd, 8, 8>(hi, lo, t, v);
        else
            tcd::WriteRowK<tc::ALayoutStd, 16, 16>(hi, lo, t, v);
    }
    else if (t < K)
    {
        for (int m0 = 0; m0 < 128; m0 += 8)
        {
            float v[8];
            for (int u = 0; u < 8; ++u)
                v[u] = A[(m0 + u) * K + t];
            if (colw == 1)
                tcd::WriteColK<tc::ALayoutStd, 8, true>(hi, lo, m0, t, v, t % 8);
            else
                tcd::WriteColK<tc::ALayoutPad, 8, false>(hi, lo, m0, t, v, 0);
        }
    }
    if (t == 0)
        MbarInit(&bar, 1);
    if (warp == 0)
        tc::Alloc(&slot, 64);
    tc::FenceProxyAsync();
    tc::FenceBeforeSync();
    __syncthreads();
    tc::FenceAfterSync();
    const uint32_t tmem = slot;
    if (t == 0)
    {
        tc::FenceAfterSync();
        if (colw == 2)
            tcd::IssuePair<tc::ALayoutPad>(tc::SmemU32(hi), 2 * tc::ALayoutPad::STEP,
                                           tc::SmemU32(sb), n, 0, n, ks, tmem, false);
        else
            tcd::IssuePair<tc::ALayoutStd>(tc::SmemU32(hi), 2 * tc::ALayoutStd::STEP,
                                           tc::SmemU32(sb), n, 0, n, ks, tmem, false);
        tc::Commit(&bar);
    }
    const bool ok = MbarWaitBounded(&bar, 0, err, 3);
    tc::FenceAfterSync();
    const uint32_t tl = tmem + (uint32_t((warp & 3) * 32) << 16);
    for (int c = 0; c < n; c += 16)
    {
        float v[16];
        tc::Ld16(tl + c, v);
        tc::WaitLd();
        for (int j = 0; j < 16; ++j)
            D[t * n + c + j] = v[j];
    }
    if (t == 0)
    {
        info[0] = tmem;
        info[1] = ok ? 1u : 0u;
    }
    tc::FenceBeforeSync();
    __syncthreads();
    if (warp == 0)
    {
        tc::FenceAfterSync();
        tc::Dealloc(tmem, 64);
    }
}
} // namespace
} // namespace nkb

using namespace nkb;

extern "C" int nkb_tc_selftest(int column_writer, int n, int ksteps, const float *A, const float *B,
                               float *D, unsigned *info)
{
    ClearError();
    if (!A || !B || !D || !info || (ksteps != 1 && ksteps != 2) ||
        (n != 16 && n != 32 && n != 64) || column_writer < 0 || column_writer > 2)
        return SetError(NKB_ERR_INVALID, "nkb_tc_selftest: n in {16, 32, 64}, ksteps 1 or 2, "
                                         "column_writer 0..2");
    const int K  = 8 * ksteps;
    float *dA    = nullptr, *dB = nullptr, *dD = nullptr;
    unsigned *dI = nullptr;
    int *dE      = nullptr;
    auto release = [&]() {
        cudaFree(dA);
        cudaFree(dB);
        cudaFree(dD);
        cudaFree(dI);
        cudaFree(dE);
    };
    if (cudaMalloc(&dA, 128 * K * 4) != cudaSuccess || cudaMalloc(&dB, K * n * 4) != cudaSuccess ||
        cudaMalloc(&dD, 128 * n * 4) != cudaSuccess || cudaMalloc(&dI, 8) != cudaSuccess ||
        cudaMalloc(&dE, 8) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_tc_selftest: buffers");
    }
    cudaMemcpy(dA, A, 128 * K * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, K * n * 4, cudaMemcpyHostToDevice);
    cudaMemset(dD, 0, 128 * n * 4);
    cudaMemset(dI, 0, 8);
    cudaMemset(dE, 0, 8);
    k_tc_selftest<<<1, 128>>>(column_writer, n, ksteps, dA, dB, dD, dI, dE);
    cudaError_t ce = cudaDeviceSynchronize();
    if (ce == cudaSuccess)
        ce = cudaMemcpy(D, dD, 128 * n * 4, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(info, dI, 8, cudaMemcpyDeviceToHost);
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_tc_selftest: %s", cudaGetErrorString(ce));
    return NKB_OK;
}
