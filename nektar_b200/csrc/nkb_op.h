// Internal definition of the operator object behind the C ABI handle.
#pragma once

#include "nkb_generic.cuh"
#include "nkb_internal.h"

#include <cuda_runtime.h>

#include <vector>

struct nkb_op
{
    int shape = 0, optype = 0, nm = 0, nq[3] = {0, 0, 0}, ptype[3] = {0, 0, 0};
    int nelmt = 0, deformed = 0, precision = 0, device = 0;
    int nc = 0, nt = 0, ncomp = 0;
    long gstride = 0; // packed geometry stride per element (multiple of 4 values)

    // 1-D tables on the device (FP64 and FP32 copies)
    double *dB[3] = {nullptr, nullptr, nullptr};
    float *fB[3]  = {nullptr, nullptr, nullptr};
    double *dD[3] = {nullptr, nullptr, nullptr};
    float *fD[3]  = {nullptr, nullptr, nullptr};
    double *dz[3] = {nullptr, nullptr, nullptr};
    double *dw[3] = {nullptr, nullptr, nullptr}; // Radau-scaled weights
    std::vector<double> hB[3], hD[3], hz[3], hw[3];

    // geometry: raw (Collections layout) and packed per point
    double *djac = nullptr, *ddf = nullptr;
    double *geo  = nullptr; // [e][ncomp][nt], element stride gstride
    float *geo32 = nullptr;

    double lambda    = 1.0;
    double factor_lambda = 1.0; // LinearADR: the caller's eFactorLambda (lambda = -factor_lambda)
    double *dvel     = nullptr; // LinearADR: V' = (-1/lambda) V on the device, three fields
    int diff_mode    = NKB_DIFF_NONE;
    double diff[6]   = {1, 0, 1, 0, 0, 1};

    // kernel selection (nkb_hex.cu): 0 generic, >0 tuned variant
    int variant     = 0;
    int hex_variant = 0; // tuned Hex kernel variant chosen by the autotuner
    int hex_variant_gather = -1; // variant for launches that gather through a
                                 // map (timed with the system's map; -1: same)
    int gen_epb     = 0; // generic kernel: elements per CTA (0: default)
    int gen_threads = 0; // generic kernel: threads per CTA (0: default)
    void *kdata = nullptr;
    int *d_err  = nullptr; // device error word (bounded waits that gave up)
    // tensor-core Hex kernel (FP32 Hex Helmholtz): B / dB tables split into
    // TF32 high and low parts in the kernel's shared-memory layout
    float *tc_tab = nullptr;
    int tc_bytes  = 0;
    int tc_tb[3]  = {0, 0, 0}, tc_tbt[3] = {0, 0, 0};
    unsigned wait_polls = 1u << 24; // first bound of bounded waits (nkb_tma.cuh kMaxPolls)

    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void *scratch        = nullptr;
    size_t scratch_bytes = 0;
};

namespace nkb
{
// generic kernels (nkb_ops.cu)
template <typename T>
int LaunchGeneric(const nkb_op *op, const T *in, T *o0, T *o1, T *o2, const int *gmap,
                  const double *gsign, cudaStream_t s, const int *skip = nullptr,
                  const double *lambda = nullptr);
// the same with IProductWRTDerivBase's three input fields as separate arrays
// (the one-input form reads them consecutively from `in`)
template <typename T>
int LaunchGeneric3(const nkb_op *op, const T *in, const T *in1, const T *in2, T *o0, T *o1, T *o2,
                   const int *gmap, const double *gsign, cudaStream_t s,
                   const int *skip = nullptr, const double *lambda = nullptr);
// per-element dense operators (nkb_dense.cu)
int LaunchDense(const nkb_op *op, const double *in, double *out, const int *gmap,
                const double *gsign, cudaStream_t s, const int *skip);
int DenseDiag(const nkb_op *op, double *d, cudaStream_t s, double *stiff);
// dispatch: tuned kernel if selected, else generic (nkb_hex.cu)
// skip: optional device flag; when it reads nonzero the kernels return at once
// (a converged CG keeps its captured graph but stops doing work)
// lambda: optional host value overriding the operator's own Helmholtz lambda
// for this launch (systems sharing one operator with different lambdas)
template <typename T>
int LaunchOp(const nkb_op *op, const T *in, T *o0, T *o1, T *o2, const int *gmap,
             const double *gsign, cudaStream_t s, const int *skip = nullptr,
             const double *lambda = nullptr);
int ChooseKernel(nkb_op *op);
// tables of the tensor-core Hex kernel (FP32 Hex Helmholtz ops, nm 2..9)
int BuildTcTables(nkb_op *op);
// reads and clears the operator's device error word (after its work has
// completed): NKB_ERR_TIMEOUT when a bounded wait gave up, else NKB_OK
int CheckOpError(nkb_op *op);
// time the Hex variants once more with the local<-global gather a system
// uses (xin: global vector, yl: local output) and keep the fastest for
// gathered launches
int TuneHexGather(nkb_op *op, const void *xin, void *yl, const int *map, const double *sign,
                  cudaStream_t s);
// name of the kernel the operator launches (for reports)
const char *KernelName(const nkb_op *op, bool gather);
size_t GenericSmemBytes(const nkb_op *op, int elem_bytes);
void FreeKernelData(nkb_op *op);
// element Helmholtz diagonals; with d_stiff the mass part (without lambda)
// goes to d_out and the Laplacian part to d_stiff, else d_out = lambda M + L
int HelmholtzDiag(const nkb_op *op, double *d_out, cudaStream_t s, double *d_stiff = nullptr);
} // namespace nkb
