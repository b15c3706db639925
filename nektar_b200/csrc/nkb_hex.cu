// Tuned Hex Helmholtz kernel and kernel selection for the element operators.
//
// The Hex Helmholtz operator (the reference's fusedKernel3D,
// MatrixFreeOps/Helmholtz.h:549-599, in the collocation form described in
// nkb_ops.cu) for nq = nm + 1 points per direction, nm = 2..11, FP64 or FP32.
//
// Work decomposition: one thread per (i, j) column of the nq x nq slab of an
// element; the third direction k lives in registers. So the contraction over
// r in BwdTrans, d/dxi_2, its transpose and the first inner-product stage are
// register-only; the i- and j-direction contractions read shared memory with
// broadcast-friendly patterns (the k-plane of a column is shared by the
// threads of a row). EPB elements share a CTA.
//
// Data movement: the element's packed geometry (W and the six metric terms,
// 7 nq^3 values) is fetched by ONE bulk TMA copy per CTA issued before any
// arithmetic, completing on an mbarrier; it streams in while BwdTrans and the
// gradient run, and only the metric stage waits for it (bounded wait). The
// 1-D tables are staged in shared memory (D padded to nq+1 columns).
// Coefficients are read coalesced, either contiguous (Collections layout) or
// gathered through the local-to-global map (the CG matvec).
#include "nkb_op.h"
#include "nkb_tma.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

namespace nkb
{

// NKB_KERNEL=generic selects the shape-generic kernels for every operator
// (used to test both implementations against each other).
static bool ForceGeneric()
{
    const char *v = std::getenv("NKB_KERNEL");
    return v && std::strcmp(v, "generic") == 0;
}

template <typename T> struct HexArgs
{
    const T *in;
    T *out;
    const int *gmap;    // optional gather (CG): in is the global vector
    const double *gsign;
    const T *geo;       // packed [e][7][nt], element stride gstride
    long gstride;
    const T *B0, *B1, *B2, *D;
    T lambda;
    int nelmt;
    int *err;
    const int *skip;    // optional: nonzero -> nothing to do (converged CG)
};

__host__ __device__ constexpr int RoundUp(int a, int b)
{
    return (a + b - 1) / b * b;
}

template <typename T, int NQ> __host__ __device__ constexpr int HexEpb()
{
    // elements per CTA: ~90 KB of shared memory per CTA, at most 512 threads
    constexpr int per = (10 * NQ * NQ * NQ + 4) * int(sizeof(T));
    constexpr int e   = (90 * 1024) / per;
    constexpr int lim = 512 / (NQ * NQ);
    constexpr int v   = e < lim ? e : lim;
    return v < 1 ? 1 : (v > 8 ? 8 : v);
}

template <typename T, int NQ> __host__ __device__ constexpr int HexThreads()
{
    return RoundUp(HexEpb<T, NQ>() * NQ * NQ, 32);
}

template <typename T, int NM, int NQ> constexpr int HexTabBytes()
{
    return RoundUp(16 + (3 * NM * NQ + NQ * (NQ + 1)) * int(sizeof(T)), 128);
}

template <typename T, int NM, int NQ, bool GATHER>
__global__ void __launch_bounds__(HexThreads<T, NQ>()) k_hex_helm(HexArgs<T> a)
{
    constexpr int NQ2 = NQ * NQ, NQ3 = NQ2 * NQ, NC = NM * NM * NM, NQP = NQ + 1;
    constexpr int EPB = HexEpb<T, NQ>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    T *sB0        = reinterpret_cast<T *>(smem + 16);
    T *sB1        = sB0 + NM * NQ;
    T *sB2        = sB1 + NM * NQ;
    T *sD         = sB2 + NM * NQ; // sD[i*NQP + m] = D(i, m) = l_m'(z_i)
    const long GS = a.gstride;
    T *geo        = reinterpret_cast<T *>(smem + HexTabBytes<T, NM, NQ>());
    T *us         = geo + EPB * GS;
    T *v0s        = us + EPB * NQ3;
    T *v1s        = v0s + EPB * NQ3;

    const int tid = threadIdx.x;
    const long e0 = long(blockIdx.x) * EPB;
    const int ne  = int(min(long(EPB), long(a.nelmt) - e0));
    if (ne <= 0 || (a.skip && *a.skip))
        return;

    if (tid == 0)
    {
        MbarInit(bar, 1);
        const uint32_t bytes = uint32_t(ne * GS * long(sizeof(T)));
        MbarArriveExpectTx(bar, bytes);
        BulkG2S(geo, a.geo + e0 * GS, bytes, bar);
    }
    for (int t = tid; t < NM * NQ; t += blockDim.x)
    {
        sB0[t] = a.B0[t];
        sB1[t] = a.B1[t];
        sB2[t] = a.B2[t];
    }
    for (int t = tid; t < NQ2; t += blockDim.x)
    {
        const int r = t / NQ, c = t - r * NQ;
        sD[r * NQP + c] = a.D[c * NQ + r];
    }
    // coefficients into the v0 region (element stride NQ3 >= NC)
    for (int t = tid; t < ne * NC; t += blockDim.x)
    {
        const int le  = t / NC;
        const int m   = t - le * NC;
        const long gi = (e0 + le) * NC + m;
        T v;
        if (GATHER)
        {
            v = a.in[a.gmap[gi]];
            if (a.gsign)
                v *= T(a.gsign[gi]);
        }
        else
        {
            v = a.in[gi];
        }
        v0s[le * NQ3 + m] = v;
    }
    __syncthreads();

    const int le   = tid / NQ2;
    const int ij   = tid - le * NQ2;
    const int i    = ij % NQ, j = ij / NQ;
    bool act       = le < ne;
    const int eoff = (le < EPB ? le : 0) * NQ3;
    T *xs = v0s + eoff, *As = v1s + eoff, *u_ = us + eoff, *v0 = v0s + eoff, *v1 = v1s + eoff;

    // BwdTrans, contraction over p: A[r][q][i], thread (i, q = j)
    if (act && j < NM)
    {
        T b0[NM];
#pragma unroll
        for (int p = 0; p < NM; ++p)
            b0[p] = sB0[p * NQ + i];
#pragma unroll
        for (int r = 0; r < NM; ++r)
        {
            const T *xr = xs + (r * NM + j) * NM;
            T s         = 0;
#pragma unroll
            for (int p = 0; p < NM; ++p)
                s = fma(xr[p], b0[p], s);
            As[(r * NM + j) * NQ + i] = s;
        }
    }
    __syncthreads();

    // contraction over q (shared memory) then over r (registers): u[k] at (i, j)
    T ur[NQ];
    if (act)
    {
        T b1[NM], bv[NM];
#pragma unroll
        for (int q = 0; q < NM; ++q)
            b1[q] = sB1[q * NQ + j];
#pragma unroll
        for (int r = 0; r < NM; ++r)
        {
            T s = 0;
#pragma unroll
            for (int q = 0; q < NM; ++q)
                s = fma(As[(r * NM + q) * NQ + i], b1[q], s);
            bv[r] = s;
        }
#pragma unroll
        for (int k = 0; k < NQ; ++k)
        {
            T s = 0;
#pragma unroll
            for (int r = 0; r < NM; ++r)
                s = fma(sB2[r * NQ + k], bv[r], s);
            ur[k]                     = s;
            u_[(k * NQ + j) * NQ + i] = s;
        }
    }
    __syncthreads();

    // geometry must have landed: bounded wait by every thread
    if (!MbarWaitBounded(bar, 0, a.err, 1))
        act = false;

    // gradient (i, j from shared memory, k from registers) and metric:
    // v = G' grad u (v0, v1 to shared memory, v2 kept), f = lambda W u
    T v2r[NQ], fr[NQ];
    if (act)
    {
        T d0[NQ], d1[NQ];
#pragma unroll
        for (int m = 0; m < NQ; ++m)
        {
            d0[m] = sD[i * NQP + m];
            d1[m] = sD[j * NQP + m];
        }
        const T *G = geo + (le < EPB ? le : 0) * GS;
#pragma unroll
        for (int k = 0; k < NQ; ++k)
        {
            T g0 = 0, g1 = 0, g2 = 0;
            const T *row = u_ + (k * NQ + j) * NQ;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                g0 = fma(d0[m], row[m], g0);
            const T *col = u_ + k * NQ2 + i;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                g1 = fma(d1[m], col[m * NQ], g1);
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                g2 = fma(sD[k * NQP + m], ur[m], g2);
            const int q = (k * NQ + j) * NQ + i;
            const T W = G[q], G00 = G[NQ3 + q], G11 = G[2 * NQ3 + q], G22 = G[3 * NQ3 + q];
            const T G01 = G[4 * NQ3 + q], G02 = G[5 * NQ3 + q], G12 = G[6 * NQ3 + q];
            v0[q]  = fma(G02, g2, fma(G01, g1, G00 * g0));
            v1[q]  = fma(G12, g2, fma(G11, g1, G01 * g0));
            v2r[k] = fma(G22, g2, fma(G12, g1, G02 * g0));
            fr[k]  = a.lambda * W * ur[k];
        }
    }
    __syncthreads();

    // f += sum_a D_a^T v_a
    if (act)
    {
        T dt0[NQ], dt1[NQ];
#pragma unroll
        for (int m = 0; m < NQ; ++m)
        {
            dt0[m] = sD[m * NQP + i];
            dt1[m] = sD[m * NQP + j];
        }
#pragma unroll
        for (int k = 0; k < NQ; ++k)
        {
            T s          = fr[k];
            const T *row = v0 + (k * NQ + j) * NQ;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                s = fma(dt0[m], row[m], s);
            const T *col = v1 + k * NQ2 + i;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                s = fma(dt1[m], col[m * NQ], s);
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                s = fma(sD[m * NQP + k], v2r[m], s);
            fr[k] = s;
        }
    }
    __syncthreads();

    // raw inner product, contraction over k (registers): T1[r][j][i] in the u region
    if (act)
    {
#pragma unroll
        for (int r = 0; r < NM; ++r)
        {
            T s = 0;
#pragma unroll
            for (int k = 0; k < NQ; ++k)
                s = fma(sB2[r * NQ + k], fr[k], s);
            u_[(r * NQ + j) * NQ + i] = s;
        }
    }
    __syncthreads();

    // contraction over j: T2[r][q][i], thread (i, q = j), into the v0 region
    if (act && j < NM)
    {
        T b1c[NQ];
#pragma unroll
        for (int jj = 0; jj < NQ; ++jj)
            b1c[jj] = sB1[j * NQ + jj];
#pragma unroll
        for (int r = 0; r < NM; ++r)
        {
            T s = 0;
#pragma unroll
            for (int jj = 0; jj < NQ; ++jj)
                s = fma(b1c[jj], u_[(r * NQ + jj) * NQ + i], s);
            v0[(r * NM + j) * NQ + i] = s;
        }
    }
    __syncthreads();

    // contraction over i: y[r][q][p], thread (p = i, q = j); coalesced stores
    if (act && i < NM && j < NM)
    {
        T b0c[NQ];
#pragma unroll
        for (int ii = 0; ii < NQ; ++ii)
            b0c[ii] = sB0[i * NQ + ii];
        T *o = a.out + (e0 + le) * NC;
#pragma unroll
        for (int r = 0; r < NM; ++r)
        {
            const T *t2 = v0 + (r * NM + j) * NQ;
            T s         = 0;
#pragma unroll
            for (int ii = 0; ii < NQ; ++ii)
                s = fma(b0c[ii], t2[ii], s);
            o[(r * NM + j) * NM + i] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

enum
{
    kVariantGeneric = 0,
    kVariantHexHelm = 1
};

template <typename T, int NM> static size_t HexSmemBytes(long gstride)
{
    constexpr int NQ = NM + 1;
    return size_t(HexTabBytes<T, NM, NQ>()) +
           size_t(HexEpb<T, NQ>()) * (size_t(gstride) + 3 * NQ * NQ * NQ) * sizeof(T);
}

template <typename T, int NM> static int HexSetAttr(long gstride)
{
    constexpr int NQ   = NM + 1;
    const size_t bytes = HexSmemBytes<T, NM>(gstride);
    if (bytes > 227 * 1024)
        return SetError(NKB_ERR_UNSUPPORTED, "tuned Hex kernel nm=%d needs %zu bytes of shared memory",
                        NM, bytes);
    NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm<T, NM, NQ, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm<T, NM, NQ, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    return NKB_OK;
}

template <typename T, int NM>
static int HexLaunch(const nkb_op *op, const HexArgs<T> &a, bool gather, cudaStream_t s)
{
    constexpr int NQ   = NM + 1;
    constexpr int EPB  = HexEpb<T, NQ>();
    const size_t bytes = HexSmemBytes<T, NM>(op->gstride);
    const long nb      = (long(op->nelmt) + EPB - 1) / EPB;
    if (nb == 0)
        return NKB_OK;
    if (gather)
        k_hex_helm<T, NM, NQ, true><<<unsigned(nb), HexThreads<T, NQ>(), bytes, s>>>(a);
    else
        k_hex_helm<T, NM, NQ, false><<<unsigned(nb), HexThreads<T, NQ>(), bytes, s>>>(a);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

#define NKB_HEX_SWITCH(NMV, CALL)                                                                  \
    switch (NMV)                                                                                   \
    {                                                                                              \
        case 2: return CALL(2);                                                                    \
        case 3: return CALL(3);                                                                    \
        case 4: return CALL(4);                                                                    \
        case 5: return CALL(5);                                                                    \
        case 6: return CALL(6);                                                                    \
        case 7: return CALL(7);                                                                    \
        case 8: return CALL(8);                                                                    \
        case 9: return CALL(9);                                                                    \
        case 10: return CALL(10);                                                                  \
        case 11: return CALL(11);                                                                  \
        default: return SetError(NKB_ERR_UNSUPPORTED, "no tuned Hex kernel for nm=%d", NMV);        \
    }

template <typename T> static int HexSetAttrT(int nm, long gstride)
{
#define NKB_CALL(N) HexSetAttr<T, N>(gstride)
    NKB_HEX_SWITCH(nm, NKB_CALL)
#undef NKB_CALL
}

template <typename T>
static int HexLaunchT(const nkb_op *op, const HexArgs<T> &a, bool gather, cudaStream_t s)
{
#define NKB_CALL(N) HexLaunch<T, N>(op, a, gather, s)
    NKB_HEX_SWITCH(op->nm, NKB_CALL)
#undef NKB_CALL
}

static bool SameTable(const std::vector<double> &a, const std::vector<double> &b)
{
    return a.size() == b.size() && std::equal(a.begin(), a.end(), b.begin());
}

int ChooseKernel(nkb_op *op)
{
    op->variant  = kVariantGeneric;
    const int eb = op->precision == NKB_FP64 ? 8 : 4;
    if (op->shape == NKB_HEX && op->optype == NKB_HELMHOLTZ && op->nm >= 2 && op->nm <= 11 &&
        op->nq[0] == op->nm + 1 && op->nq[1] == op->nq[0] && op->nq[2] == op->nq[0] &&
        SameTable(op->hD[0], op->hD[1]) && SameTable(op->hD[0], op->hD[2]) && !ForceGeneric())
    {
        int rc = op->precision == NKB_FP64 ? HexSetAttrT<double>(op->nm, op->gstride)
                                           : HexSetAttrT<float>(op->nm, op->gstride);
        if (rc == NKB_OK)
        {
            op->variant = kVariantHexHelm;
            return NKB_OK;
        }
        ClearError();
    }
    if (GenericSmemBytes(op, eb) > 200 * 1024)
        return SetError(NKB_ERR_UNSUPPORTED,
                        "nkb_op_create: nm=%d nq=(%d,%d,%d) needs %zu bytes of shared memory per "
                        "element", op->nm, op->nq[0], op->nq[1], op->nq[2], GenericSmemBytes(op, eb));
    return NKB_OK;
}

void FreeKernelData(nkb_op *op)
{
    op->kdata = nullptr;
}

template <typename T>
int LaunchOp(const nkb_op *op, const T *in, T *o0, T *o1, T *o2, const int *gmap,
             const double *gsign, cudaStream_t s, const int *skip)
{
    if (op->variant == kVariantHexHelm)
    {
        HexArgs<T> a;
        a.in      = in;
        a.out     = o0;
        a.gmap    = gmap;
        a.gsign   = gsign;
        a.geo     = std::is_same<T, double>::value ? (const T *)op->geo : (const T *)op->geo32;
        a.gstride = op->gstride;
        const void *const *B = std::is_same<T, double>::value ? (const void *const *)op->dB
                                                               : (const void *const *)op->fB;
        const void *const *D = std::is_same<T, double>::value ? (const void *const *)op->dD
                                                               : (const void *const *)op->fD;
        a.B0     = (const T *)B[0];
        a.B1     = (const T *)B[1];
        a.B2     = (const T *)B[2];
        a.D      = (const T *)D[0];
        a.lambda = T(op->lambda);
        a.nelmt  = op->nelmt;
        a.err    = op->d_err;
        a.skip   = skip;
        return HexLaunchT<T>(op, a, gmap != nullptr, s);
    }
    return LaunchGeneric<T>(op, in, o0, o1, o2, gmap, gsign, s, skip);
}

template int LaunchOp<double>(const nkb_op *, const double *, double *, double *, double *,
                              const int *, const double *, cudaStream_t, const int *);
template int LaunchOp<float>(const nkb_op *, const float *, float *, float *, float *,
                             const int *, const double *, cudaStream_t, const int *);

} // namespace nkb
