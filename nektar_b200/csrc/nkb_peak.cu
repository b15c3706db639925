// Arithmetic peaks of the device measured in place, the compute denominators
// of the operators' rooflines (a copy bandwidth and a BF16 GEMM rate are
// measured elsewhere; FP64 and FP32 rates are not): FP64 fused multiply-add
// on the CUDA cores, FP64 tensor-core MMA (mma.sync m8n8k4), FP32 fused
// multiply-add. Every thread runs independent dependency chains, so the
// timed rate is the pipe's throughput, not its latency.
#include "nkb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>

namespace nkb
{
namespace
{
constexpr int kPeakThreads = 256;
constexpr int kChains      = 8;

template <typename T> __global__ void __launch_bounds__(kPeakThreads) k_fma_peak(int iters, T *out)
{
    T a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        a[c] = T(1) + T(threadIdx.x + c) * T(1e-3);
    const T m = T(0.999999), b = T(1e-7); // the chains stay bounded
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            a[c] = fma(a[c], m, b);
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += a[c];
    out[blockIdx.x * long(blockDim.x) + threadIdx.x] = s; // keeps the chains live
}

constexpr int kMmaChains = 4;

__global__ void __launch_bounds__(kPeakThreads) k_dmma_peak(int iters, double *out)
{
    const int lane = threadIdx.x & 31;
    double c0[kMmaChains], c1[kMmaChains];
#pragma unroll
    for (int u = 0; u < kMmaChains; ++u)
        c0[u] = c1[u] = 0.0;
    const double a = 1e-3 * (lane + 1), b = 0.5;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int u = 0; u < kMmaChains; ++u)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
                         "{%0, %1};\n"
                         : "+d"(c0[u]), "+d"(c1[u])
                         : "d"(a), "d"(b));
    double s = 0.0;
#pragma unroll
    for (int u = 0; u < kMmaChains; ++u)
        s += c0[u] + c1[u];
    out[blockIdx.x * long(blockDim.x) + threadIdx.x] = s;
}
} // namespace
} // namespace nkb

using namespace nkb;

extern "C" int nkb_peak_probe(int kind, int device, double *tflops)
{
    ClearError();
    if (!tflops || kind < 0 || kind > 2)
        return SetError(NKB_ERR_INVALID, "nkb_peak_probe: kind 0 (FP64 FMA), 1 (FP64 MMA) or "
                                         "2 (FP32 FMA)");
    NKB_CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    NKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid     = sms * 8;
    const long threads = long(grid) * kPeakThreads;
    const int iters    = kind == 1 ? 2048 : 8192;
    // flops of one launch: FMA 2 per chain step; MMA 2 * 8 * 8 * 4 per warp step
    const double flops = kind == 1 ? 2.0 * 8 * 8 * 4 * kMmaChains * double(iters) * (threads / 32)
                                   : 2.0 * kChains * double(iters) * threads;
    void *out      = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&]() {
        cudaFree(out);
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
        if (s)
            cudaStreamDestroy(s);
    };
    // one value per launched thread (doubles: room for either type)
    if (cudaMalloc(&out, threads * sizeof(double)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_peak_probe: buffers");
    }
    auto launch = [&]() {
        if (kind == 0)
            k_fma_peak<double><<<grid, kPeakThreads, 0, s>>>(iters, static_cast<double *>(out));
        else if (kind == 1)
            k_dmma_peak<<<grid, kPeakThreads, 0, s>>>(iters, static_cast<double *>(out));
        else
            k_fma_peak<float><<<grid, kPeakThreads, 0, s>>>(iters, static_cast<float *>(out));
    };
    double best    = 0.0;
    cudaError_t ce = cudaSuccess;
    for (int r = 0; r < 8 && ce == cudaSuccess; ++r)
    {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        ce = cudaGetLastError();
        if (ce == cudaSuccess)
            ce = cudaEventSynchronize(e1);
        float ms = 0.f;
        // the first three launches warm up
        if (ce == cudaSuccess && r >= 3 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0)
            best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_peak_probe: %s", cudaGetErrorString(ce));
    *tflops = best;
    return NKB_OK;
}
