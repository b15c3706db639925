// Per-element dense operators: y_e = M_e x_e for nelmt blocks of rows x cols
// matrices. Used for the statically condensed (boundary) system of
// GlobalLinSysIterativeStaticCond (MultiRegions/GlobalLinSysIterativeStaticCond
// .cpp, GlobalLinSysStaticCond.cpp: the Schur complement of each element's
// Helmholtz matrix on its boundary modes, applied element by element and
// assembled). The operator plugs into a CG system like a Helmholtz
// collection: gathered launches read x through the local -> global map, its
// diagonal feeds the Jacobi preconditioner.
//
// The matrices are the whole data stream (n^2 doubles per element), so the
// kernel is a batched, HBM-bound GEMV: one CTA per element, the element's
// input staged in shared memory, each warp reading whole rows with
// coalesced loads and reducing them with a fixed shuffle tree (the result
// does not depend on the launch).
#include "nkb_internal.h"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <cstring>

namespace nkb
{

constexpr int kDenseThreads = 256;

template <bool GATHER>
__global__ void __launch_bounds__(kDenseThreads)
    k_dense_gemv(const double *__restrict__ M, int rows, int cols, long nelmt,
                 const double *__restrict__ x, const int *__restrict__ gmap,
                 const double *__restrict__ gsign, double *__restrict__ y, const int *skip)
{
    extern __shared__ double xs[];
    const long e = blockIdx.x;
    if (e >= nelmt || (skip && *skip))
        return;
    for (int j = threadIdx.x; j < cols; j += blockDim.x)
    {
        const long l = e * cols + j;
        if (GATHER)
            xs[j] = gsign ? gsign[l] * x[gmap[l]] : x[gmap[l]];
        else
            xs[j] = x[l];
    }
    __syncthreads();
    const double *Me = M + e * long(rows) * cols;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < rows; i += kDenseThreads / 32)
    {
        const double *row = Me + long(i) * cols;
        double s = 0.0;
        for (int j = lane; j < cols; j += 32)
            s = fma(__ldg(row + j), xs[j], s);
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
            y[e * rows + i] = s;
    }
}

__global__ void k_dense_diag(const double *__restrict__ M, int n, long nelmt, double *d,
                             double *zero)
{
    const long tot = nelmt * n;
    for (long g = blockIdx.x * long(blockDim.x) + threadIdx.x; g < tot;
         g += long(gridDim.x) * blockDim.x)
    {
        const long e = g / n, i = g % n;
        d[g] = M[(e * n + i) * n + i];
        if (zero)
            zero[g] = 0.0;
    }
}

int LaunchDense(const nkb_op *op, const double *in, double *out, const int *gmap,
                const double *gsign, cudaStream_t s, const int *skip)
{
    if (op->nelmt == 0)
        return NKB_OK;
    // rows = op->nt outputs and cols = op->nc inputs per element
    const size_t smem = size_t(op->nc) * sizeof(double);
    if (gmap)
        k_dense_gemv<true><<<unsigned(op->nelmt), kDenseThreads, smem, s>>>(
            op->geo, op->nt, op->nc, op->nelmt, in, gmap, gsign, out, skip);
    else
        k_dense_gemv<false><<<unsigned(op->nelmt), kDenseThreads, smem, s>>>(
            op->geo, op->nt, op->nc, op->nelmt, in, nullptr, nullptr, out, skip);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

// diagonal of every block; with `stiff`, the blocks' diagonal goes there and
// `d` (the mass part of a Helmholtz split) is zero
int DenseDiag(const nkb_op *op, double *d, cudaStream_t s, double *stiff)
{
    const long tot = long(op->nelmt) * op->nc;
    if (op->nc != op->nt)
        return SetError(NKB_ERR_INVALID, "diagonal of non-square dense blocks");
    if (tot == 0)
        return NKB_OK;
    const int nb = int(std::min<long>((tot + 255) / 256, 148L * 16));
    if (stiff)
        k_dense_diag<<<nb, 256, 0, s>>>(op->geo, op->nc, op->nelmt, stiff, d);
    else
        k_dense_diag<<<nb, 256, 0, s>>>(op->geo, op->nc, op->nelmt, d, nullptr);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

} // namespace nkb

using namespace nkb;

extern "C" int nkb_op_create_dense_rect(int rows, int cols, int nelmt, const double *mats,
                                        int device, nkb_op **out)
{
    ClearError();
    if (!out || (!mats && nelmt > 0) || rows < 1 || cols < 1 || nelmt < 0)
        return SetError(NKB_ERR_INVALID, "nkb_op_create_dense: bad arguments");
    *out = nullptr;
    if (size_t(cols) * sizeof(double) > 48 * 1024)
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_op_create_dense: blocks of %d columns", cols);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return SetError(NKB_ERR_NO_DEVICE, "nkb_op_create_dense: no CUDA device");
    if (device < 0 || device >= ndev)
        return SetError(NKB_ERR_INVALID, "nkb_op_create_dense: device %d of %d", device, ndev);
    NKB_CUDA_TRY(cudaSetDevice(device));
    nkb_op *op    = new nkb_op();
    op->optype    = NKB_DENSE_BLOCK;
    op->nelmt     = nelmt;
    op->nc        = cols;
    op->nt        = rows;
    op->precision = NKB_FP64;
    op->device    = device;
    op->lambda    = 1.0;
    auto fail = [&](int code) {
        nkb_op_destroy(op);
        return code;
    };
    if (cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&op->ev0) != cudaSuccess || cudaEventCreate(&op->ev1) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_op_create_dense: stream/event creation failed"));
    if (cudaMalloc(&op->d_err, 2 * sizeof(int)) != cudaSuccess ||
        cudaMemset(op->d_err, 0, 2 * sizeof(int)) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_op_create_dense: error word"));
    const size_t bytes = size_t(nelmt) * rows * cols * sizeof(double);
    if (bytes)
    {
        if (cudaMalloc(&op->geo, bytes) != cudaSuccess)
            return fail(SetError(NKB_ERR_NOMEM, "nkb_op_create_dense: %zu bytes of blocks", bytes));
        // host or device blocks (unified addressing tells them apart)
        // a copy from device memory does not wait for itself: finished here,
        // so the caller may free the source on return
        if (cudaMemcpy(op->geo, mats, bytes, cudaMemcpyDefault) != cudaSuccess ||
            cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess)
            return fail(SetError(NKB_ERR_CUDA, "nkb_op_create_dense: upload"));
    }
    *out = op;
    return NKB_OK;
}

extern "C" int nkb_op_create_dense(int n, int nelmt, const double *mats, int device,
                                   nkb_op **out)
{
    return nkb_op_create_dense_rect(n, n, nelmt, mats, device, out);
}
