// nkb_op_apply_host_static: the host-pointer operator apply without any
// device allocation.
//
// nkb_op_apply(..., NKB_HOST_PTRS, ...) stages the caller's host arrays in a
// device buffer it allocates (and grows) with cudaMalloc. Some callers cannot
// allocate device memory at the point where they apply an operator: a solver
// that reserved the device memory it may use at start-up and must stay inside
// that budget, or a time-stepping loop that must not pay the device-wide
// synchronisation cudaMalloc / cudaFree can cause. For them this file keeps
// the staging area in a fixed, file-scope device array instead:
//
//   * size: NKB_STATIC_SCRATCH_DOUBLES doubles (32 MiB), held by every GPU
//     that loads the library until the process exits;
//   * an operator fits when its input plus all its outputs fit in it
//     (nkb_op_sizes: in + out, or in + 3 out for PhysDeriv); larger operators
//     are rejected with NKB_ERR_INVALID;
//   * the device address of the array is looked up once per device, on the
//     first call made on that device (cudaGetSymbolAddress with that device
//     current); make that first call before capturing any stream;
//   * every call uses the same array, so calls whose work overlaps on the GPU
//     (different host threads or streams at the same time) race: serialise
//     them. Nothing in the array needs to start at zero: each call writes the
//     whole input and the kernels write every output value before the copy
//     back.
#include "nkb_internal.h"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <mutex>

#define NKB_STATIC_SCRATCH_DOUBLES (4L * 1024L * 1024L)

static __device__ __align__(256) double g_nkb_static_scratch[NKB_STATIC_SCRATCH_DOUBLES];

namespace
{
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double *g_static_ptr[kMaxDevices] = {};

// device address of the static array on `device` (which must be current)
int StaticScratch(int device, double **out)
{
    if (device < 0 || device >= kMaxDevices)
        return nkb::SetError(NKB_ERR_INVALID, "nkb_op_apply_host_static: device %d", device);
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[device])
    {
        void *p        = nullptr;
        cudaError_t ce = cudaGetSymbolAddress(&p, g_nkb_static_scratch);
        if (ce != cudaSuccess || !p)
            return nkb::SetError(NKB_ERR_CUDA,
                                 "nkb_op_apply_host_static: cudaGetSymbolAddress failed: %s",
                                 cudaGetErrorString(ce));
        g_static_ptr[device] = static_cast<double *>(p);
    }
    *out = g_static_ptr[device];
    return NKB_OK;
}
} // namespace

using namespace nkb;

// the staged apply on the operator's device (current)
static int ApplyStatic(nkb_op *op, const double *in, double *out0, double *out1, double *out2,
                       long nin, long nout, int nouts, cudaStream_t s)
{
    double *scratch = nullptr;
    int rc          = StaticScratch(op->device, &scratch);
    if (rc)
        return rc;
    double *din  = scratch;
    double *dout = scratch + nin;
    NKB_CUDA_TRY(cudaMemcpyAsync(din, in, nin * sizeof(double), cudaMemcpyHostToDevice, s));
    rc = LaunchOp<double>(op, din, dout, nouts > 1 ? dout + nout : nullptr,
                          nouts > 2 ? dout + 2 * nout : nullptr, nullptr, nullptr, s);
    if (rc)
        return rc;
    double *outs[3] = {out0, out1, out2};
    for (int o = 0; o < nouts; ++o)
        NKB_CUDA_TRY(cudaMemcpyAsync(outs[o], dout + o * nout, nout * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    return CheckOpError(op);
}

extern "C" int nkb_op_apply_host_static(nkb_op *op, const double *in, double *out0, double *out1,
                                        double *out2, void *stream)
{
    ClearError();
    if (!op || !in || !out0)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply_host_static: NULL argument");
    if (op->precision != NKB_FP64)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply_host_static: needs an FP64 operator");
    const int nouts = op->optype == NKB_PHYSDERIV ? 3 : 1;
    if (nouts == 3 && (!out1 || !out2))
        return SetError(NKB_ERR_INVALID, "nkb_op_apply_host_static: PhysDeriv needs three outputs");
    long nin = 0, nout = 0;
    int rc = nkb_op_sizes(op, &nin, &nout);
    if (rc)
        return rc;
    const long need = nin + nouts * nout;
    if (need > NKB_STATIC_SCRATCH_DOUBLES)
        return SetError(NKB_ERR_INVALID,
                        "nkb_op_apply_host_static: operator needs %ld doubles of staging, the "
                        "static area holds %ld (32 MiB); use nkb_op_apply",
                        need, (long)NKB_STATIC_SCRATCH_DOUBLES);
    // the operator's device is made current for the call; the caller's
    // current device is restored on every return
    int caller_dev = 0;
    NKB_CUDA_TRY(cudaGetDevice(&caller_dev));
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    rc = ApplyStatic(op, in, out0, out1, out2, nin, nout, nouts, static_cast<cudaStream_t>(stream));
    const cudaError_t ce = cudaSetDevice(caller_dev);
    if (rc)
        return rc;
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_op_apply_host_static: restoring device %d: %s",
                        caller_dev, cudaGetErrorString(ce));
    return NKB_OK;
}
