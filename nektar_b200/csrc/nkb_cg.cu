// Global Helmholtz system and its preconditioned conjugate gradient on the
// device: GlobalLinSysIterativeFull (MultiRegions/GlobalLinSysIterativeFull.cpp
// :96-384) with PreconditionerDiagonal (PreconditionerDiagonal.cpp:93-189)
// over AssemblyMapCG (AssemblyMap/AssemblyMapCG.cpp:2772-2906), driving the
// reduced-communication PCG of NekLinSysIterCG::DoConjugateGradient
// (LinearAlgebra/NekLinSysIterCG.cpp:118-372).
//
// One CG iteration is four launches that never return to the host:
//   k_update    p = w + beta p; q = s + beta q; x += alpha p; r -= alpha q;
//               w = diag^-1 r; block partials of (r,w) and (r,r)
//   operators   gather w through the local->global map inside the element
//               kernel, element Helmholtz, local result
//   k_assemble  s = Assemble(local) as a gather over a global->local CSR
//               (deterministic, no atomics) + block partials of (s,w)
//   k_scalars   fixed-order reduction of the partials, convergence test
//               eps < tol^2 |b|^2, new alpha / beta; sets done
// Scalars stay on the device; the host polls "done" once per block of
// check_interval iterations, which can be captured as a CUDA graph.
#include "nkb_internal.h"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace nkb
{

struct CGState
{
    double rho, mu, eps, alpha, beta;
    double rhs_mag, tol2;
    int iter, maxit, done, status;
};

static constexpr int kRedBlocks = 1184; // 148 SMs x 8
static constexpr int kRedThreads = 256;

__device__ __forceinline__ double WarpSum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block sum of two values into part[blockIdx.x*2 + {0,1}]
__device__ __forceinline__ void BlockSum2(double a, double b, double *part)
{
    __shared__ double sa[32], sb[32];
    a = WarpSum(a);
    b = WarpSum(b);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
    {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (warp == 0)
    {
        const int nw = blockDim.x >> 5;
        a            = lane < nw ? sa[lane] : 0.0;
        b            = lane < nw ? sb[lane] : 0.0;
        a            = WarpSum(a);
        b            = WarpSum(b);
        if (lane == 0)
        {
            part[2 * blockIdx.x]     = a;
            part[2 * blockIdx.x + 1] = b;
        }
    }
}

template <typename T>
__global__ void k_update(int nn, int ndir, const CGState *st, T *__restrict__ p, T *__restrict__ q,
                         T *__restrict__ x, T *__restrict__ r, T *__restrict__ w,
                         const T *__restrict__ s, const T *__restrict__ dinv, double *part)
{
    if (st->done)
        return;
    const T beta = T(st->beta), alpha = T(st->alpha);
    double rw = 0.0, rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const T pi = fma(beta, p[i], w[ndir + i]);
        const T qi = fma(beta, q[i], s[ndir + i]);
        p[i]       = pi;
        q[i]       = qi;
        x[ndir + i] = fma(alpha, pi, x[ndir + i]);
        const T ri = fma(-alpha, qi, r[i]);
        r[i]       = ri;
        const T wi = ri * dinv[i];
        w[ndir + i] = wi;
        rw += double(ri) * double(wi);
        rr += double(ri) * double(ri);
    }
    BlockSum2(rw, rr, part);
}

// w = diag^-1 r on the non-Dirichlet part, with (r,w) and (r,r) partials
template <typename T>
__global__ void k_precon(int nn, int ndir, const CGState *st, const T *__restrict__ r,
                         T *__restrict__ w, const T *__restrict__ dinv, double *part)
{
    if (st->done)
        return;
    double rw = 0.0, rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const T wi = r[i] * dinv[i];
        w[ndir + i] = wi;
        rw += double(r[i]) * double(wi);
        rr += double(r[i]) * double(r[i]);
    }
    BlockSum2(rw, rr, part);
}

template <typename T>
__global__ void k_assemble(int nglob, int ndir, const int *__restrict__ aptr,
                           const int *__restrict__ aidx, const double *__restrict__ sign,
                           const T *__restrict__ loc, T *__restrict__ glob,
                           const T *__restrict__ w, const CGState *st, double *part)
{
    if (st && st->done)
        return;
    double sw = 0.0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nglob; g += gridDim.x * blockDim.x)
    {
        T acc = 0;
        const int k1 = aptr[g + 1];
        for (int k = aptr[g]; k < k1; ++k)
        {
            const int l = aidx[k];
            acc += sign ? T(sign[l]) * loc[l] : loc[l];
        }
        glob[g] = acc;
        if (w && g >= ndir)
            sw += double(acc) * double(w[g]);
    }
    if (part)
        BlockSum2(sw, 0.0, part);
}

__global__ void k_global_to_local(long nloc, const int *__restrict__ map,
                                  const double *__restrict__ sign, const double *__restrict__ glob,
                                  double *__restrict__ loc)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < nloc;
         i += long(gridDim.x) * blockDim.x)
        loc[i] = sign ? sign[i] * glob[map[i]] : glob[map[i]];
}

// fixed-order sum of the first (even: 0, odd: 1) entries of nb partial pairs
__device__ double ReducePart(const double *part, int nb, int which)
{
    __shared__ double red[1024];
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        v += part[2 * b + which];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    double out = red[0];
    __syncthreads();
    return out;
}

// mode 0: initial residual: eps = (r,r) from partA[1], rhs_mag = (b,b) from partB[0]
// mode 1: first direction:  rho = (r,w) partA[0], mu = (s,w) partB[0]; alpha = rho/mu
// mode 2: iteration:        rho_new, eps from partA, mu from partB
__global__ void k_scalars(CGState *st, const double *partA, int nbA, const double *partB, int nbB,
                          int mode)
{
    if (st->done)
        return;
    const double a0 = ReducePart(partA, nbA, 0);
    const double a1 = ReducePart(partA, nbA, 1);
    const double b0 = ReducePart(partB, nbB, 0);
    if (threadIdx.x != 0)
        return;
    if (mode == 0)
    {
        st->eps     = a1;
        double rhs  = b0;
        st->rhs_mag = rhs > 1.0e-6 ? rhs : 1.0; // NekLinSysIter.cpp:96-117
        st->iter    = 0;
        if (!(st->eps < st->tol2 * st->rhs_mag))
            return;
        st->done   = 1;
        st->status = NKB_OK;
        return;
    }
    if (mode == 1)
    {
        st->rho   = a0;
        st->mu    = b0;
        st->beta  = 0.0;
        st->alpha = a0 / b0;
        st->iter  = 1;
        if (!isfinite(st->alpha))
        {
            st->done   = 1;
            st->status = NKB_ERR_NONFINITE;
        }
        return;
    }
    const double rho_new = a0, eps = a1, mu = b0;
    st->mu  = mu;
    st->eps = eps;
    st->iter += 1;
    if (eps < st->tol2 * st->rhs_mag)
    {
        st->done   = 1;
        st->status = NKB_OK;
        return;
    }
    const double beta  = rho_new / st->rho;
    const double alpha = rho_new / (mu - rho_new * beta / st->alpha);
    st->beta           = beta;
    st->alpha          = alpha;
    st->rho            = rho_new;
    if (!isfinite(alpha) || !isfinite(eps))
    {
        st->done   = 1;
        st->status = NKB_ERR_NONFINITE;
        return;
    }
    if (st->iter > st->maxit)
    {
        st->done   = 1;
        st->status = NKB_ERR_NOT_CONVERGED;
    }
}

__global__ void k_init(int nglob, int ndir, const double *__restrict__ bglob, double *r, double *x,
                       double *w, double *s, double *p, double *q, double *part)
{
    double rr = 0.0, bb = 0.0;
    const int nn = nglob - ndir;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nglob; g += gridDim.x * blockDim.x)
    {
        const double b = bglob[g];
        bb += b * b;
        x[g] = 0.0;
        w[g] = 0.0;
        s[g] = 0.0;
        if (g >= ndir)
        {
            r[g - ndir] = b;
            p[g - ndir] = 0.0;
            q[g - ndir] = 0.0;
            rr += b * b;
        }
    }
    (void)nn;
    BlockSum2(bb, rr, part);
}

__global__ void k_axpy_loc(long n, double a, const double *__restrict__ xv, double *__restrict__ y)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        y[i] = fma(a, xv[i], y[i]);
}

__global__ void k_sub_loc(long n, const double *__restrict__ a, const double *__restrict__ b,
                          double *__restrict__ out)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        out[i] = a[i] - b[i];
}

__global__ void k_invert(int nn, int ndir, const double *__restrict__ dglob, double *__restrict__ dinv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        dinv[i] = 1.0 / dglob[ndir + i];
}

// ---- mixed precision (FP64 iterative refinement around an FP32 PCG) --------

// inner solve start: r32 = (float) r64, x32 = w32 = s32 = p32 = q32 = 0, partial (r,r)
__global__ void k_init_inner(int nglob, int ndir, const double *__restrict__ r64,
                             float *__restrict__ r32, float *__restrict__ x32,
                             float *__restrict__ w32, float *__restrict__ s32,
                             float *__restrict__ p32, float *__restrict__ q32, double *part)
{
    double rr = 0.0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nglob; g += gridDim.x * blockDim.x)
    {
        x32[g] = 0.f;
        w32[g] = 0.f;
        s32[g] = 0.f;
        if (g >= ndir)
        {
            const float r   = float(r64[g - ndir]);
            r32[g - ndir] = r;
            p32[g - ndir] = 0.f;
            q32[g - ndir] = 0.f;
            rr += double(r) * double(r);
        }
    }
    BlockSum2(0.0, rr, part);
}

// x64 += x32 on the non-Dirichlet part
__global__ void k_add_correction(int nn, int ndir, double *__restrict__ x64,
                                 const float *__restrict__ x32)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        x64[ndir + i] += double(x32[ndir + i]);
}

// r = b - s on the non-Dirichlet part (s = A x assembled), partial (r,r)
__global__ void k_residual(int nn, int ndir, const double *__restrict__ b, const double *__restrict__ s,
                           double *__restrict__ r, double *part)
{
    double rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const double v = b[ndir + i] - s[ndir + i];
        r[i]           = v;
        rr += v * v;
    }
    BlockSum2(0.0, rr, part);
}

// start of an inner solve: eps = (r,r) = rhs_mag (relative criterion), iter = 0
__global__ void k_scalars_inner_init(CGState *st, const double *part, int nb, double tol2,
                                     int maxit)
{
    const double rr = ReducePart(part, nb, 1);
    if (threadIdx.x != 0)
        return;
    st->eps     = rr;
    st->rhs_mag = rr > 0.0 ? rr : 1.0;
    st->tol2    = tol2;
    st->maxit   = maxit;
    st->iter    = 0;
    st->status  = NKB_OK;
    st->done    = (rr > 0.0) ? 0 : 1;
}

// outer residual norm into st->eps
__global__ void k_scalars_outer(CGState *st, const double *part, int nb)
{
    const double rr = ReducePart(part, nb, 1);
    if (threadIdx.x == 0)
        st->eps = rr;
}

__global__ void k_float_copy(long n, const double *__restrict__ a, float *__restrict__ b)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        b[i] = float(a[i]);
}

static int Blocks(long n, int threads = kRedThreads)
{
    return int(std::max<long>(1, std::min<long>((n + threads - 1) / threads, kRedBlocks)));
}

} // namespace nkb

using namespace nkb;

struct nkb_sys
{
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<nkb_op *> ops;
    std::vector<long> off;
    long nloc = 0;
    int nglob = 0, ndir = 0, nn = 0;
    int *d_map = nullptr;
    double *d_sign = nullptr;
    int *d_aptr = nullptr, *d_aidx = nullptr;
    double *d_dinv = nullptr;
    double *w = nullptr, *s = nullptr, *x = nullptr, *p = nullptr, *r = nullptr, *q = nullptr;
    double *bglob = nullptr, *yl = nullptr, *tl = nullptr;
    double *partA = nullptr, *partB = nullptr;
    CGState *st = nullptr;
    CGState *h_st = nullptr; // pinned
    cudaGraphExec_t graph = nullptr;
    int graph_k = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double *stage = nullptr; // host-pointer staging (2*nloc)
    long launches = 0;       // kernels launched by the current solve
    // mixed precision: FP32 twins of the operators and the inner-CG state
    std::vector<nkb_op *> ops32;
    float *w32 = nullptr, *s32 = nullptr, *x32 = nullptr, *p32 = nullptr, *r32 = nullptr,
          *q32 = nullptr, *yl32 = nullptr, *dinv32 = nullptr;
    CGState *st32 = nullptr;
    cudaGraphExec_t graph32 = nullptr;
    int graph32_k = 0;
};

namespace nkb
{

// y_loc = A x_loc over all collections; x given either as a local vector or
// as a global vector gathered through the map (gather = true).
static int Matvec(nkb_sys *S, const double *xin, double *yl, bool gather, cudaStream_t s,
                  const int *skip = nullptr)
{
    for (size_t c = 0; c < S->ops.size(); ++c)
    {
        const nkb_op *op = S->ops[c];
        const long o     = S->off[c];
        int rc;
        if (gather)
            rc = LaunchOp<double>(op, xin, yl + o, nullptr, nullptr, S->d_map + o,
                                  S->d_sign ? S->d_sign + o : nullptr, s, skip);
        else
            rc = LaunchOp<double>(op, xin + o, yl + o, nullptr, nullptr, nullptr, nullptr, s, skip);
        if (rc)
            return rc;
    }
    return NKB_OK;
}

static int Matvec32(nkb_sys *S, const float *xin, float *yl, cudaStream_t s, const int *skip)
{
    for (size_t c = 0; c < S->ops32.size(); ++c)
    {
        const long o = S->off[c];
        int rc = LaunchOp<float>(S->ops32[c], xin, yl + o, nullptr, nullptr, S->d_map + o,
                                 S->d_sign ? S->d_sign + o : nullptr, s, skip);
        if (rc)
            return rc;
    }
    return NKB_OK;
}

// one FP32 inner-CG iteration (same recurrence as Iteration, FP64 dot sums)
static int Iteration32(nkb_sys *S, cudaStream_t s)
{
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    S->launches += 3 + long(S->ops32.size());
    k_update<float><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st32, S->p32, S->q32, S->x32,
                                                S->r32, S->w32, S->s32, S->dinv32, S->partA);
    int rc = Matvec32(S, S->w32, S->yl32, s, &S->st32->done);
    if (rc)
        return rc;
    k_assemble<float><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                  S->d_sign, S->yl32, S->s32, S->w32, S->st32,
                                                  S->partB);
    k_scalars<<<1, 1024, 0, s>>>(S->st32, S->partA, nbU, S->partB, nbA, 2);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

static int Iteration(nkb_sys *S, cudaStream_t s)
{
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    S->launches += 3 + long(S->ops.size());
    k_update<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->p, S->q, S->x, S->r,
                                                 S->w, S->s, S->d_dinv, S->partA);
    int rc = Matvec(S, S->w, S->yl, true, s, &S->st->done);
    if (rc)
        return rc;
    k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                   S->d_sign, S->yl, S->s, S->w, S->st, S->partB);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbU, S->partB, nbA, 2);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

} // namespace nkb

extern "C" int nkb_sys_create(const nkb_sys_desc *desc, nkb_sys **out)
{
    ClearError();
    if (!desc || !out || !desc->ops || desc->nops < 1 || !desc->map)
        return SetError(NKB_ERR_INVALID, "nkb_sys_create: bad arguments");
    *out = nullptr;
    long nloc = 0;
    for (int c = 0; c < desc->nops; ++c)
    {
        const nkb_op *op = desc->ops[c];
        if (!op || op->optype != NKB_HELMHOLTZ || op->precision != NKB_FP64)
            return SetError(NKB_ERR_INVALID, "nkb_sys_create: op %d is not an FP64 Helmholtz op", c);
        nloc += long(op->nelmt) * op->nc;
    }
    if (nloc != desc->nloc)
        return SetError(NKB_ERR_INVALID, "nkb_sys_create: nloc %ld != sum of collections %ld",
                        desc->nloc, nloc);
    if (desc->nglob < 1 || desc->ndir < 0 || desc->ndir > desc->nglob)
        return SetError(NKB_ERR_INVALID, "nkb_sys_create: nglob=%d ndir=%d", desc->nglob, desc->ndir);
    for (long i = 0; i < nloc; ++i)
        if (desc->map[i] < 0 || desc->map[i] >= desc->nglob)
            return SetError(NKB_ERR_INVALID, "nkb_sys_create: map[%ld]=%d outside [0,%d)", i,
                            desc->map[i], desc->nglob);
    NKB_CUDA_TRY(cudaSetDevice(desc->device));
    nkb_sys *S = new nkb_sys();
    auto fail  = [&](int code) {
        nkb_sys_destroy(S);
        return code;
    };
    S->device = desc->device;
    S->nloc   = nloc;
    S->nglob  = desc->nglob;
    S->ndir   = desc->ndir;
    S->nn     = desc->nglob - desc->ndir;
    long o    = 0;
    for (int c = 0; c < desc->nops; ++c)
    {
        S->ops.push_back(desc->ops[c]);
        S->off.push_back(o);
        o += long(desc->ops[c]->nelmt) * desc->ops[c]->nc;
    }
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&S->ev0) != cudaSuccess || cudaEventCreate(&S->ev1) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_sys_create: stream/event"));

    // global -> local CSR for the deterministic assemble
    std::vector<int> aptr(S->nglob + 1, 0), aidx(nloc);
    for (long i = 0; i < nloc; ++i)
        aptr[desc->map[i] + 1]++;
    for (int g = 0; g < S->nglob; ++g)
        aptr[g + 1] += aptr[g];
    {
        std::vector<int> fill(aptr.begin(), aptr.end() - 1);
        for (long i = 0; i < nloc; ++i)
            aidx[fill[desc->map[i]]++] = int(i);
    }
    auto dalloc = [&](void **ptr, size_t bytes) -> bool {
        return cudaMalloc(ptr, std::max<size_t>(bytes, 8)) == cudaSuccess;
    };
    bool ok = dalloc((void **)&S->d_map, nloc * sizeof(int)) &&
              dalloc((void **)&S->d_aptr, (S->nglob + 1) * sizeof(int)) &&
              dalloc((void **)&S->d_aidx, nloc * sizeof(int)) &&
              dalloc((void **)&S->d_dinv, S->nn * sizeof(double)) &&
              dalloc((void **)&S->w, S->nglob * sizeof(double)) &&
              dalloc((void **)&S->s, S->nglob * sizeof(double)) &&
              dalloc((void **)&S->x, S->nglob * sizeof(double)) &&
              dalloc((void **)&S->bglob, S->nglob * sizeof(double)) &&
              dalloc((void **)&S->p, S->nn * sizeof(double)) &&
              dalloc((void **)&S->r, S->nn * sizeof(double)) &&
              dalloc((void **)&S->q, S->nn * sizeof(double)) &&
              dalloc((void **)&S->yl, nloc * sizeof(double)) &&
              dalloc((void **)&S->tl, nloc * sizeof(double)) &&
              dalloc((void **)&S->partA, 2 * kRedBlocks * sizeof(double)) &&
              dalloc((void **)&S->partB, 2 * kRedBlocks * sizeof(double)) &&
              dalloc((void **)&S->st, sizeof(CGState));
    if (!ok)
        return fail(SetError(NKB_ERR_NOMEM, "nkb_sys_create: device allocation failed"));
    if (cudaMallocHost(&S->h_st, sizeof(CGState)) != cudaSuccess)
        return fail(SetError(NKB_ERR_NOMEM, "nkb_sys_create: pinned state"));
    if (desc->ops32)
    {
        for (int c = 0; c < desc->nops; ++c)
        {
            const nkb_op *a = desc->ops[c], *b = desc->ops32[c];
            if (!b || b->optype != NKB_HELMHOLTZ || b->precision != NKB_FP32 ||
                b->nelmt != a->nelmt || b->nc != a->nc)
                return fail(SetError(NKB_ERR_INVALID,
                                     "nkb_sys_create: ops32[%d] is not an FP32 twin of ops[%d]", c,
                                     c));
            S->ops32.push_back(desc->ops32[c]);
        }
        bool ok32 = dalloc((void **)&S->w32, S->nglob * sizeof(float)) &&
                    dalloc((void **)&S->s32, S->nglob * sizeof(float)) &&
                    dalloc((void **)&S->x32, S->nglob * sizeof(float)) &&
                    dalloc((void **)&S->p32, S->nn * sizeof(float)) &&
                    dalloc((void **)&S->r32, S->nn * sizeof(float)) &&
                    dalloc((void **)&S->q32, S->nn * sizeof(float)) &&
                    dalloc((void **)&S->dinv32, S->nn * sizeof(float)) &&
                    dalloc((void **)&S->yl32, nloc * sizeof(float)) &&
                    dalloc((void **)&S->st32, sizeof(CGState));
        if (!ok32)
            return fail(SetError(NKB_ERR_NOMEM, "nkb_sys_create: FP32 vectors"));
    }
    NKB_CUDA_TRY(cudaMemcpy(S->d_map, desc->map, nloc * sizeof(int), cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaMemcpy(S->d_aptr, aptr.data(), (S->nglob + 1) * sizeof(int), cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaMemcpy(S->d_aidx, aidx.data(), nloc * sizeof(int), cudaMemcpyHostToDevice));
    if (desc->sign)
    {
        if (!dalloc((void **)&S->d_sign, nloc * sizeof(double)))
            return fail(SetError(NKB_ERR_NOMEM, "nkb_sys_create: sign"));
        NKB_CUDA_TRY(cudaMemcpy(S->d_sign, desc->sign, nloc * sizeof(double), cudaMemcpyHostToDevice));
    }
    // Jacobi diagonal: element diagonals, assembled, inverted
    // (PreconditionerDiagonal::DiagonalPreconditionerSum, :93-125)
    for (size_t c = 0; c < S->ops.size(); ++c)
    {
        int rc = HelmholtzDiag(S->ops[c], S->tl + S->off[c], S->stream);
        if (rc)
            return fail(rc);
    }
    // sign^2 = 1: the diagonal sums the raw local entries
    k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, S->stream>>>(
        S->nglob, S->ndir, S->d_aptr, S->d_aidx, nullptr, S->tl, S->bglob, nullptr, nullptr, nullptr);
    k_invert<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(S->nn, S->ndir, S->bglob, S->d_dinv);
    if (S->dinv32)
        k_float_copy<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(S->nn, S->d_dinv, S->dinv32);
    NKB_CUDA_TRY(cudaGetLastError());
    NKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    *out = S;
    return NKB_OK;
}

extern "C" int nkb_sys_diag_inv(nkb_sys *S, double *diag_inv, int flags, void *stream)
{
    if (!S || !diag_inv)
        return SetError(NKB_ERR_INVALID, "nkb_sys_diag_inv: NULL argument");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    NKB_CUDA_TRY(cudaMemcpyAsync(diag_inv, S->d_dinv, S->nn * sizeof(double),
                                 (flags & NKB_HOST_PTRS) ? cudaMemcpyDeviceToHost
                                                         : cudaMemcpyDeviceToDevice,
                                 s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    return NKB_OK;
}

extern "C" int nkb_sys_assemble(nkb_sys *S, const double *loc, double *glob, void *stream)
{
    if (!S || !loc || !glob)
        return SetError(NKB_ERR_INVALID, "nkb_sys_assemble: NULL argument");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
        S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, loc, glob, nullptr, nullptr, nullptr);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

extern "C" int nkb_sys_global_to_local(nkb_sys *S, const double *glob, double *loc, void *stream)
{
    if (!S || !loc || !glob)
        return SetError(NKB_ERR_INVALID, "nkb_sys_global_to_local: NULL argument");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    k_global_to_local<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, S->d_map, S->d_sign, glob, loc);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

extern "C" int nkb_sys_matvec_local(nkb_sys *S, const double *x_loc, double *y_loc, void *stream)
{
    if (!S || !x_loc || !y_loc)
        return SetError(NKB_ERR_INVALID, "nkb_sys_matvec_local: NULL argument");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    return Matvec(S, x_loc, y_loc, false, s);
}

namespace nkb
{
// FP64 iterative refinement around an FP32 PCG, on the lifted system (bglob
// already assembled): r = b - A x in FP64, an FP32 PCG solves A d = r to a
// relative reduction inner_tol (FP64 sums of the dot products), x += d in
// FP64, until ||r||^2 < tol^2 ||b||^2 (NekLinSysIterCG's criterion). The
// geometry, the residual, the norms and the solution stay FP64; S->st ends
// with the FP64 residual and the total inner iteration count.
static int MixedSolve(nkb_sys *S, const nkb_cg_opts &o, cudaStream_t s, int *outer_out)
{
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    const int K   = o.check_interval;
    const double tol       = std::fmax(o.tol, 1.0e-16);
    const double inner_tol = o.inner_tol > 0 ? o.inner_tol : 1.0e-5;
    const int max_outer    = o.max_outer > 0 ? o.max_outer : 40;
    CGState h0;
    std::memset(&h0, 0, sizeof(h0));
    h0.tol2  = tol * tol;
    h0.maxit = o.maxit;
    NKB_CUDA_TRY(cudaMemcpyAsync(S->st, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    k_init<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->bglob, S->r, S->x, S->w, S->s, S->p,
                                       S->q, S->partA);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbA, S->partA, nbA, 0);
    S->launches += 2;
    if (S->graph32 == nullptr || S->graph32_k != K)
    {
        if (S->graph32)
            cudaGraphExecDestroy(S->graph32);
        S->graph32 = nullptr;
        cudaGraph_t g;
        NKB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int crc = NKB_OK;
        for (int k = 0; k < K && !crc; ++k)
            crc = Iteration32(S, s);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        S->launches -= long(K) * (3 + long(S->ops32.size()));
        if (crc)
            return crc;
        if (ce != cudaSuccess)
            return SetError(NKB_ERR_CUDA, "mixed CG graph capture: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&S->graph32, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess)
            return SetError(NKB_ERR_CUDA, "mixed CG graph instantiate: %s", cudaGetErrorString(ce));
        S->graph32_k = K;
    }
    int total = 0, outer = 0, rc = NKB_OK;
    CGState h, h32;
    for (; outer <= max_outer; ++outer)
    {
        NKB_CUDA_TRY(cudaMemcpyAsync(&h, S->st, sizeof(h), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        if (!std::isfinite(h.eps))
        {
            h.done   = 1;
            h.status = NKB_ERR_NONFINITE;
            break;
        }
        if (h.done || h.eps < h.tol2 * h.rhs_mag)
        {
            h.done   = 1;
            h.status = NKB_OK;
            break;
        }
        if (outer == max_outer || total >= o.maxit)
        {
            h.done   = 1;
            h.status = NKB_ERR_NOT_CONVERGED;
            break;
        }
        // inner FP32 PCG on A d = r
        k_init_inner<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->r, S->r32, S->x32, S->w32,
                                                 S->s32, S->p32, S->q32, S->partA);
        k_scalars_inner_init<<<1, 1024, 0, s>>>(S->st32, S->partA, nbA, inner_tol * inner_tol,
                                                o.maxit - total);
        k_precon<float><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st32, S->r32, S->w32,
                                                    S->dinv32, S->partA);
        if ((rc = Matvec32(S, S->w32, S->yl32, s, &S->st32->done)))
            return rc;
        k_assemble<float><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                      S->d_sign, S->yl32, S->s32, S->w32, S->st32,
                                                      S->partB);
        k_scalars<<<1, 1024, 0, s>>>(S->st32, S->partA, nbU, S->partB, nbA, 1);
        S->launches += 6 + long(S->ops32.size());
        const int max_passes = (o.maxit - total) / K + 2;
        for (int pass = 0; pass < max_passes; ++pass)
        {
            NKB_CUDA_TRY(cudaMemcpyAsync(&h32, S->st32, sizeof(h32), cudaMemcpyDeviceToHost, s));
            NKB_CUDA_TRY(cudaStreamSynchronize(s));
            if (h32.done)
                break;
            NKB_CUDA_TRY(cudaGraphLaunch(S->graph32, s));
            S->launches += long(K) * (3 + long(S->ops32.size()));
        }
        NKB_CUDA_TRY(cudaMemcpyAsync(&h32, S->st32, sizeof(h32), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        total += std::max(h32.iter, 1);
        // x += d; r = b - A x and its norm, all FP64
        k_add_correction<<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->x, S->x32);
        if ((rc = Matvec(S, S->x, S->yl, true, s)))
            return rc;
        k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                       S->d_sign, S->yl, S->s, nullptr, nullptr,
                                                       nullptr);
        k_residual<<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->bglob, S->s, S->r, S->partA);
        k_scalars_outer<<<1, 1024, 0, s>>>(S->st, S->partA, nbU);
        S->launches += 4 + long(S->ops.size());
        NKB_CUDA_TRY(cudaGetLastError());
    }
    h.iter = total;
    NKB_CUDA_TRY(cudaMemcpyAsync(S->st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    *outer_out = outer;
    return NKB_OK;
}
} // namespace nkb

extern "C" int nkb_cg_solve(nkb_sys *S, const double *b_loc, double *x_loc,
                            const nkb_cg_opts *opts, nkb_cg_report *rep, int flags, void *stream)
{
    ClearError();
    if (!S || !b_loc || !x_loc)
        return SetError(NKB_ERR_INVALID, "nkb_cg_solve: NULL argument");
    nkb_cg_opts o;
    std::memset(&o, 0, sizeof(o));
    o.tol            = 1e-9;
    o.maxit          = 5000;
    o.check_interval = 16;
    o.use_graph      = 1;
    if (opts)
        o = *opts;
    if (o.tol <= 0)
        o.tol = 1e-9;
    if (o.maxit <= 0)
        o.maxit = 5000;
    if (o.check_interval <= 0)
        o.check_interval = 16;
    if (o.mixed && S->ops32.empty())
        return SetError(NKB_ERR_INVALID, "nkb_cg_solve: mixed precision needs FP32 operators "
                                         "(nkb_sys_desc.ops32)");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    // NULL (or the legacy default stream) -> the system's own stream
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    const long nloc = S->nloc;

    const double *db = b_loc;
    double *dx       = x_loc;
    if (flags & NKB_HOST_PTRS)
    {
        if (!S->stage && cudaMalloc(&S->stage, 2 * nloc * sizeof(double)) != cudaSuccess)
            return SetError(NKB_ERR_NOMEM, "nkb_cg_solve: staging buffers");
        NKB_CUDA_TRY(cudaMemcpyAsync(S->stage, b_loc, nloc * sizeof(double), cudaMemcpyHostToDevice, s));
        NKB_CUDA_TRY(cudaMemcpyAsync(S->stage + nloc, x_loc, nloc * sizeof(double), cudaMemcpyHostToDevice, s));
        db = S->stage;
        dx = S->stage + nloc;
    }
    NKB_CUDA_TRY(cudaEventRecord(S->ev0, s));
    S->launches = 0;

    // Dirichlet lifting (GlobalLinSysIterativeFull.cpp:104-164):
    // rhs = b - A x_D (local), gloIn = Assemble(rhs)
    int rc = Matvec(S, dx, S->yl, false, s);
    if (rc)
        return rc;
    k_sub_loc<<<Blocks(nloc), kRedThreads, 0, s>>>(nloc, db, S->yl, S->tl);
    k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
        S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, S->tl, S->bglob, nullptr, nullptr, nullptr);

    int outer_done = 0;
    if (o.mixed)
    {
        if ((rc = MixedSolve(S, o, s, &outer_done)))
            return rc;
        goto finish;
    }
    {
    CGState h0;
    std::memset(&h0, 0, sizeof(h0));
    const double tol = std::fmax(o.tol, 1.0e-16); // NekLinSysIter.cpp:57
    h0.tol2          = tol * tol;
    h0.maxit         = o.maxit;
    NKB_CUDA_TRY(cudaMemcpyAsync(S->st, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    k_init<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->bglob, S->r, S->x, S->w, S->s, S->p,
                                       S->q, S->partA);
    // partA holds (b,b) in [0] and (r,r) in [1]; k_scalars mode 0 reads eps
    // from partA[1] and rhs from partB[0]
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbA, S->partA, nbA, 0);
    k_precon<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->r, S->w, S->d_dinv, S->partA);
    if ((rc = Matvec(S, S->w, S->yl, true, s)))
        return rc;
    k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                   S->d_sign, S->yl, S->s, S->w, S->st, S->partB);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbU, S->partB, nbA, 1);
    NKB_CUDA_TRY(cudaGetLastError());
    // lift (ops + sub + assemble), init, scalars, precon, ops, assemble, scalars
    S->launches += 2 * long(S->ops.size()) + 7;

    const int K = o.check_interval;
    bool use_graph = o.use_graph != 0;
    if (use_graph && (S->graph == nullptr || S->graph_k != K))
    {
        if (S->graph)
        {
            cudaGraphExecDestroy(S->graph);
            S->graph = nullptr;
        }
        if (s != cudaStreamLegacy && s != cudaStreamPerThread)
        {
            cudaGraph_t g;
            NKB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            int crc = NKB_OK;
            for (int k = 0; k < K && !crc; ++k)
                crc = Iteration(S, s);
            cudaError_t ce = cudaStreamEndCapture(s, &g);
            if (crc)
                return crc;
            if (ce != cudaSuccess)
                return SetError(NKB_ERR_CUDA, "nkb_cg_solve: graph capture: %s", cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&S->graph, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess)
                return SetError(NKB_ERR_CUDA, "nkb_cg_solve: graph instantiate: %s", cudaGetErrorString(ce));
            S->graph_k = K;
            S->launches -= long(K) * (3 + long(S->ops.size())); // captured, not launched
        }
        else
        {
            use_graph = false; // caller stream: launch directly
        }
    }
    // iterate until the device reports done; each pass runs K iterations
    // (kernels are no-ops once done is set)
    const int max_passes = o.maxit / K + 2;
    for (int pass = 0; pass < max_passes; ++pass)
    {
        NKB_CUDA_TRY(cudaMemcpyAsync(S->h_st, S->st, sizeof(CGState), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        if (S->h_st->done)
            break;
        if (use_graph)
        {
            NKB_CUDA_TRY(cudaGraphLaunch(S->graph, s));
            S->launches += long(K) * (3 + long(S->ops.size()));
        }
        else
        {
            for (int k = 0; k < K; ++k)
                if ((rc = Iteration(S, s)))
                    return rc;
        }
    }
    }
finish:
    NKB_CUDA_TRY(cudaMemcpyAsync(S->h_st, S->st, sizeof(CGState), cudaMemcpyDeviceToHost, s));
    // x_loc += GlobalToLocal(x) (the Dirichlet part of x is zero)
    k_global_to_local<<<Blocks(nloc), kRedThreads, 0, s>>>(nloc, S->d_map, S->d_sign, S->x, S->tl);
    k_axpy_loc<<<Blocks(nloc), kRedThreads, 0, s>>>(nloc, 1.0, S->tl, dx);
    S->launches += 2;
    NKB_CUDA_TRY(cudaEventRecord(S->ev1, s));
    if (flags & NKB_HOST_PTRS)
        NKB_CUDA_TRY(cudaMemcpyAsync(x_loc, dx, nloc * sizeof(double), cudaMemcpyDeviceToHost, s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    const CGState &h = *S->h_st;
    if (rep)
    {
        rep->iterations       = h.iter;
        rep->outer_iterations = outer_done;
        rep->rel_residual     = std::sqrt(h.eps / h.rhs_mag);
        rep->converged        = (h.done && h.status == NKB_OK) ? 1 : 0;
        float ms              = 0.f;
        cudaEventElapsedTime(&ms, S->ev0, S->ev1);
        rep->device_ms       = ms;
        rep->kernel_launches = S->launches;
    }
    if (h.status == NKB_ERR_NONFINITE)
        return SetError(NKB_ERR_NONFINITE, "nkb_cg_solve: non-finite CG scalar at iteration %d", h.iter);
    if (h.status == NKB_ERR_NOT_CONVERGED || !h.done)
        return SetError(NKB_ERR_NOT_CONVERGED,
                        "nkb_cg_solve: CG iterations made = %d exceeded maxit (error = %g)", h.iter,
                        std::sqrt(h.eps / h.rhs_mag));
    return NKB_OK;
}

extern "C" int nkb_sys_profile_iteration(nkb_sys *S, int iters, nkb_sys_profile *prof)
{
    ClearError();
    if (!S || !prof || iters < 1)
        return SetError(NKB_ERR_INVALID, "nkb_sys_profile_iteration: bad arguments");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t s = S->stream;
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    cudaEvent_t e[5];
    for (auto &ev : e)
        NKB_CUDA_TRY(cudaEventCreate(&ev));
    // the kernels read the live state; make sure they run (done = 0) on a copy
    CGState h;
    NKB_CUDA_TRY(cudaMemcpy(&h, S->st, sizeof(h), cudaMemcpyDeviceToHost));
    CGState run = h;
    run.done    = 0;
    run.maxit   = 1 << 30;
    NKB_CUDA_TRY(cudaMemcpy(S->st, &run, sizeof(run), cudaMemcpyHostToDevice));
    int rc = NKB_OK;
    NKB_CUDA_TRY(cudaEventRecord(e[0], s));
    for (int it = 0; it < iters && !rc; ++it)
        rc = Matvec(S, S->w, S->yl, true, s);
    NKB_CUDA_TRY(cudaEventRecord(e[1], s));
    for (int it = 0; it < iters; ++it)
        k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                       S->d_sign, S->yl, S->s, S->w, S->st,
                                                       S->partB);
    NKB_CUDA_TRY(cudaEventRecord(e[2], s));
    // the update kernel with alpha = beta = 0 leaves x unchanged and w = dinv r
    CGState zero = run;
    zero.alpha = zero.beta = 0.0;
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    NKB_CUDA_TRY(cudaMemcpy(S->st, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaEventRecord(e[2], s));
    for (int it = 0; it < iters; ++it)
        k_update<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->p, S->q, S->x,
                                                     S->r, S->w, S->s, S->d_dinv, S->partA);
    NKB_CUDA_TRY(cudaEventRecord(e[3], s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    cudaEvent_t e4, e5;
    NKB_CUDA_TRY(cudaEventCreate(&e4));
    NKB_CUDA_TRY(cudaEventCreate(&e5));
    NKB_CUDA_TRY(cudaEventRecord(e4, s));
    for (int it = 0; it < iters; ++it)
        k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbU, S->partB, nbA, 2);
    NKB_CUDA_TRY(cudaEventRecord(e5, s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    NKB_CUDA_TRY(cudaGetLastError());
    float t01 = 0, t12 = 0, t23 = 0, t45 = 0;
    cudaEventElapsedTime(&t01, e[0], e[1]);
    cudaEventElapsedTime(&t12, e[1], e[2]);
    cudaEventElapsedTime(&t23, e[2], e[3]);
    cudaEventElapsedTime(&t45, e4, e5);
    for (auto &ev : e)
        cudaEventDestroy(ev);
    cudaEventDestroy(e4);
    cudaEventDestroy(e5);
    // restore the state of the last solve
    NKB_CUDA_TRY(cudaMemcpy(S->st, &h, sizeof(h), cudaMemcpyHostToDevice));
    if (rc)
        return rc;
    prof->op_ms       = t01 / iters;
    prof->assemble_ms = t12 / iters;
    prof->update_ms   = t23 / iters;
    prof->scalars_ms  = t45 / iters;
    double bytes = 0.0, flops = 0.0;
    for (const nkb_op *op : S->ops)
    {
        const double nq = op->nq[0], nm = op->nm;
        // geometry (7 values per point), coefficients in through the int32
        // map, coefficients out
        bytes += double(op->nelmt) * (8.0 * 7.0 * op->nt + 20.0 * op->nc);
        if (op->shape == NKB_HEX)
            flops += double(op->nelmt) *
                     (4.0 * (nq * nm * nm * nm + nq * nq * nm * nm + nq * nq * nq * nm) +
                      12.0 * nq * nq * nq * nq + 18.0 * nq * nq * nq);
    }
    prof->op_bytes = bytes;
    prof->op_flops = flops;
    return NKB_OK;
}

extern "C" void nkb_sys_destroy(nkb_sys *S)
{
    if (!S)
        return;
    cudaSetDevice(S->device);
    if (S->graph)
        cudaGraphExecDestroy(S->graph);
    if (S->graph32)
        cudaGraphExecDestroy(S->graph32);
    for (void *ptr : {(void *)S->w32, (void *)S->s32, (void *)S->x32, (void *)S->p32,
                      (void *)S->r32, (void *)S->q32, (void *)S->dinv32, (void *)S->yl32,
                      (void *)S->st32})
        cudaFree(ptr);
    cudaFree(S->d_map);
    cudaFree(S->d_sign);
    cudaFree(S->d_aptr);
    cudaFree(S->d_aidx);
    cudaFree(S->d_dinv);
    cudaFree(S->w);
    cudaFree(S->s);
    cudaFree(S->x);
    cudaFree(S->bglob);
    cudaFree(S->p);
    cudaFree(S->r);
    cudaFree(S->q);
    cudaFree(S->yl);
    cudaFree(S->tl);
    cudaFree(S->partA);
    cudaFree(S->partB);
    cudaFree(S->st);
    cudaFree(S->stage);
    if (S->h_st)
        cudaFreeHost(S->h_st);
    if (S->ev0)
        cudaEventDestroy(S->ev0);
    if (S->ev1)
        cudaEventDestroy(S->ev1);
    if (S->stream)
        cudaStreamDestroy(S->stream);
    delete S;
}
