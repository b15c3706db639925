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
// check_interval iterations, which can be captured as a CUDA graph. The solve
// is a non-blocking state machine (nkb_cg_begin / nkb_cg_poll / nkb_cg_end), so
// one host thread can keep many systems' solves in flight on their own streams;
// nkb_cg_solve polls it with waits. Clones (nkb_sys_clone) share operators, map
// and diagonal and own their vectors, and may each carry their own lambda.
#include "nkb_internal.h"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
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

// the partial dot products count the free dofs i < nown only (all of them on
// one GPU; a shard's own dofs, numbered first, in a sharded solve). wjac: the
// previous w is the Jacobi step of the previous r (no block step has changed
// it), so it is recomputed as r dinv, the same product, instead of read.
template <typename T>
__global__ void k_update(int nn, int ndir, const CGState *st, T *__restrict__ p, T *__restrict__ q,
                         T *__restrict__ x, T *__restrict__ r, T *__restrict__ w,
                         const T *__restrict__ s, const T *__restrict__ dinv, double *part,
                         int nown, int wjac)
{
    if (st->done)
        return;
    const T beta = T(st->beta), alpha = T(st->alpha);
    double rw = 0.0, rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const T rold = r[i], dv = dinv[i];
        const T wold = wjac ? rold * dv : w[ndir + i];
        const T pi   = fma(beta, p[i], wold);
        const T qi   = fma(beta, q[i], s[ndir + i]);
        p[i]       = pi;
        q[i]       = qi;
        x[ndir + i] = fma(alpha, pi, x[ndir + i]);
        const T ri = fma(-alpha, qi, rold);
        r[i]       = ri;
        const T wi = ri * dv;
        w[ndir + i] = wi;
        if (i < nown)
        {
            rw += double(ri) * double(wi);
            rr += double(ri) * double(ri);
        }
    }
    BlockSum2(rw, rr, part);
}

// w = diag^-1 r on the non-Dirichlet part, with (r,w) and (r,r) partials
// over the free dofs i < nown
template <typename T>
__global__ void k_precon(int nn, int ndir, const CGState *st, const T *__restrict__ r,
                         T *__restrict__ w, const T *__restrict__ dinv, double *part, int nown)
{
    if (st->done)
        return;
    double rw = 0.0, rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const T wi = r[i] * dinv[i];
        w[ndir + i] = wi;
        if (i < nown)
        {
            rw += double(r[i]) * double(wi);
            rr += double(r[i]) * double(r[i]);
        }
    }
    BlockSum2(rw, rr, part);
}

// Block-Jacobi step (PreconditionerBlock::v_DoPreconditioner,
// PreconditionerBlock.cpp; PreconditionerLowEnergy::v_DoPreconditioner,
// PreconditionerLowEnergy.cpp:915-933): for every block b of dofs idx_b, w_b =
// M_b^-1 r_b, replacing the diagonal step's w there. One warp per block and
// a grid of one CTA per 8 blocks (all blocks in flight at once: the step is
// latency-bound, a few MB of blocks), the inverse stored column-major so a
// warp's lanes read consecutive rows. The change of (r,w) goes to per-CTA
// partials that k_scalars adds to (r,w) in a fixed order.
constexpr int kBlockMax     = 256; // largest block (rows)
constexpr int kBlockWarps   = kRedThreads / 32;
constexpr int kBlockGridMax = 8192;

__global__ void __launch_bounds__(kRedThreads)
    k_block_precon(int nblk, int ndir, const CGState *st, const int *__restrict__ bptr,
                   const int *__restrict__ bidx, const long *__restrict__ boff,
                   const double *__restrict__ bmat, const double *__restrict__ r,
                   double *__restrict__ w, double *part)
{
    if (st->done)
        return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double corr = 0.0;
    for (int b = blockIdx.x * kBlockWarps + warp; b < nblk; b += gridDim.x * kBlockWarps)
    {
        const int o = bptr[b], n = bptr[b + 1] - o;
        const int *idx = bidx + o;
        const double *M = bmat + boff[b];
        // rows i0 + lane; columns in chunks of 32 whose r values sit one per
        // lane (shuffled to all), so a chunk's 32 loads per lane and its r
        // gather are in flight together (the step is latency-bound)
        for (int i0 = 0; i0 < n; i0 += 32)
        {
            const int i   = i0 + lane;
            const bool ir = i < n;
            double acc = 0.0, ri = 0.0, wold = 0.0;
            long gi = 0;
            for (int j0 = 0; j0 < n; j0 += 32)
            {
                const int jl = j0 + lane;
                long gj      = 0;
                double rj    = 0.0, wj = 0.0;
                if (jl < n)
                {
                    gj = long(ndir) + idx[jl];
                    rj = r[idx[jl]];
                    if (j0 == i0)
                        wj = w[gj];
                }
                double m[32];
#pragma unroll
                for (int u = 0; u < 32; ++u)
                    m[u] = (ir && j0 + u < n) ? __ldg(M + long(j0 + u) * n + i) : 0.0;
#pragma unroll
                for (int u = 0; u < 32; ++u)
                    acc = fma(m[u], __shfl_sync(0xffffffffu, rj, u), acc);
                if (j0 == i0) // this lane's own row i = jl
                {
                    ri   = rj;
                    wold = wj;
                    gi   = gj;
                }
            }
            if (ir)
            {
                corr += ri * (acc - wold);
                w[gi] = acc;
            }
        }
    }
    __shared__ double red[kBlockWarps];
    corr = WarpSum(corr);
    if (lane == 0)
        red[warp] = corr;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        for (int k = 0; k < kBlockWarps; ++k)
            t += red[k];
        part[2 * blockIdx.x]     = t;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// glob = assembled loc; (glob, w) partial over the dofs ndir <= g < ndir + nsw
// (every free dof on one GPU; a shard's dofs that no other shard touches in a
// sharded solve, whose assembled values are complete there)
template <typename T>
__global__ void k_assemble(int nglob, int ndir, const int *__restrict__ aptr,
                           const int *__restrict__ aidx, const double *__restrict__ sign,
                           const T *__restrict__ loc, T *__restrict__ glob,
                           const T *__restrict__ w, const CGState *st, double *part, int nsw)
{
    if (st && st->done)
        return;
    // a thread's dofs g0, g0 + stride, ... are taken four at a time with their
    // entries walked in lockstep, so the index and value loads of four dofs
    // are in flight together; every dof still sums its entries in CSR order
    // and the thread visits its dofs in the same order
    constexpr int U = 4;
    const int stride = gridDim.x * blockDim.x;
    double sw        = 0.0;
    for (int g0 = blockIdx.x * blockDim.x + threadIdx.x; g0 < nglob; g0 += U * stride)
    {
        int k0[U], k1[U];
        int kmax = 0;
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int g = g0 + u * stride;
            k0[u]       = g < nglob ? aptr[g] : 0;
            k1[u]       = g < nglob ? aptr[g + 1] : 0;
            kmax        = max(kmax, k1[u] - k0[u]);
        }
        T acc[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            acc[u] = 0;
        for (int j = 0; j < kmax; ++j)
        {
            int l[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                l[u] = k0[u] + j < k1[u] ? aidx[k0[u] + j] : -1;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (l[u] >= 0)
                    acc[u] += sign ? T(sign[l[u]]) * loc[l[u]] : loc[l[u]];
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int g = g0 + u * stride;
            if (g < nglob)
            {
                glob[g] = acc[u];
                if (w && g >= ndir && g - ndir < nsw)
                    sw += double(acc[u]) * double(w[g]);
            }
        }
    }
    if (part)
        BlockSum2(sw, 0.0, part);
}

// the Jacobi diagonal: element diagonals summed per global dof, leaving out
// local modes whose sign is 0 (a mode a lower-order neighbour lacks,
// PreconditionerDiagonal::DiagonalPreconditionerSum, PreconditionerDiagonal.cpp
// :104-117)
__global__ void k_assemble_diag(int nglob, const int *__restrict__ aptr,
                                const int *__restrict__ aidx, const double *__restrict__ sign,
                                const double *__restrict__ loc, double *__restrict__ glob)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nglob; g += gridDim.x * blockDim.x)
    {
        double acc = 0.0;
        for (int k = aptr[g]; k < aptr[g + 1]; ++k)
        {
            const int l = aidx[k];
            if (!sign || sign[l] != 0.0)
                acc += loc[l];
        }
        glob[g] = acc;
    }
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
// mode 3: restart of the recurrence after a reliable update (mixed precision)
// (a0, a1, b0: the sums of partA[0], partA[1], partB[0]; one thread)
__device__ void ScalarStep(CGState *st, double a0, double a1, double b0, int mode)
{
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
    if (mode == 3)
    {
        // the residual was replaced by the true one (reliable update): new
        // rho, mu from it; beta, alpha against the last accepted rho, alpha
        // (a paused iteration did not overwrite them); iteration count kept
        const double beta  = a0 / st->rho;
        const double alpha = a0 / (b0 - a0 * beta / st->alpha);
        st->mu    = b0;
        st->eps   = a1;
        st->beta  = beta;
        st->alpha = alpha;
        st->rho   = a0;
        if (!isfinite(alpha) || !isfinite(a1))
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

// partC (nbC > 0): the block preconditioner's corrections of (r,w)
__global__ void k_scalars(CGState *st, const double *partA, int nbA, const double *partB, int nbB,
                          int mode, const double *partC = nullptr, int nbC = 0)
{
    if (st->done)
        return;
    double a0 = ReducePart(partA, nbA, 0);
    if (nbC)
        a0 += ReducePart(partC, nbC, 0);
    const double a1 = ReducePart(partA, nbA, 1);
    const double b0 = ReducePart(partB, nbB, 0);
    if (threadIdx.x != 0)
        return;
    ScalarStep(st, a0, a1, b0, mode);
}

__global__ void k_init(int nglob, int ndir, const double *__restrict__ bglob, double *r, double *x,
                       double *w, double *s, double *p, double *q, double *part,
                       const unsigned char *__restrict__ dcnt, int nown)
{
    double rr = 0.0, bb = 0.0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nglob; g += gridDim.x * blockDim.x)
    {
        const double b = bglob[g];
        x[g] = 0.0;
        w[g] = 0.0;
        s[g] = 0.0;
        if (g >= ndir)
        {
            r[g - ndir] = b;
            p[g - ndir] = 0.0;
            q[g - ndir] = 0.0;
            if (g - ndir < nown)
            {
                bb += b * b;
                rr += b * b;
            }
        }
        else if (!dcnt || dcnt[g])
            bb += b * b;
    }
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

// ---- mixed precision (FP32 PCG with FP64 reliable updates) -----------------

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

// x64 += x32 and x32 = 0 on the non-Dirichlet part (a reliable update folds
// the FP32 correction into the FP64 solution)
__global__ void k_add_correction(int nn, int ndir, double *__restrict__ x64, float *__restrict__ x32)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        x64[ndir + i] += double(x32[ndir + i]);
        x32[ndir + i] = 0.f;
    }
}

// r = b - s on the non-Dirichlet part (s = A x assembled), r32 = (float) r,
// partial (r,r)
__global__ void k_residual(int nn, int ndir, const double *__restrict__ b, const double *__restrict__ s,
                           double *__restrict__ r, float *__restrict__ r32, double *part)
{
    double rr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const double v = b[ndir + i] - s[ndir + i];
        r[i]           = v;
        r32[i]         = float(v);
        rr += v * v;
    }
    BlockSum2(0.0, rr, part);
}

// FP32 CG (re)start after a reliable update: the iterated residual pauses
// the CG once (r,r) < thr; reset = 1 also zeroes the iteration count
__global__ void k_resume(CGState *st, double thr, int maxit, int reset)
{
    st->tol2    = thr;
    st->rhs_mag = 1.0;
    st->maxit   = maxit;
    st->status  = NKB_OK;
    st->done    = 0;
    if (reset)
        st->iter = 0;
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

// Jacobi inverse for a system lambda from the split assembled diagonal:
// dinv = 1 / (lambda dM + dL) on the non-Dirichlet part (and its FP32 copy)
__global__ void k_combine_dinv(int nn, int ndir, double lambda, const double *__restrict__ dM,
                               const double *__restrict__ dL, double *__restrict__ dinv,
                               float *__restrict__ dinv32)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
    {
        const double v = 1.0 / fma(lambda, dM[ndir + i], dL[ndir + i]);
        dinv[i]        = v;
        if (dinv32)
            dinv32[i] = float(v);
    }
}

static int Blocks(long n, int threads = kRedThreads)
{
    return int(std::max<long>(1, std::min<long>((n + threads - 1) / threads, kRedBlocks)));
}

} // namespace nkb

namespace nkb
{
// What a system and its clones share: the operators, the local->global map
// with its global->local CSR and optional sign, and the split assembled
// Jacobi diagonal (mass and Laplacian parts, built on first use).
struct SysShared
{
    int device = 0;
    std::vector<nkb_op *> ops, ops32;
    std::vector<long> off;
    long nloc = 0;
    int nglob = 0, ndir = 0, nn = 0;
    int *d_map = nullptr, *d_aptr = nullptr, *d_aidx = nullptr;
    double *d_sign = nullptr;
    double *d_dM = nullptr, *d_dL = nullptr; // nglob each
    // optional block-Jacobi preconditioner (nkb_sys_set_blocks): blocks of
    // non-Dirichlet dofs with their inverses; other dofs keep Jacobi
    int nblk = 0;
    int *d_bptr = nullptr, *d_bidx = nullptr;
    long *d_boff = nullptr;
    double *d_bmat = nullptr;
    size_t bytes = 0;
    std::mutex mu; // guards the lazy split diagonal
    // a shard of a sharded group (nkb_shard_group_create): its diagonal
    // parts hold the whole mesh's values at the shared dofs, and it solves
    // only through the group
    bool grouped = false;

    ~SysShared()
    {
        cudaSetDevice(device);
        for (void *p : {(void *)d_map, (void *)d_aptr, (void *)d_aidx, (void *)d_sign,
                        (void *)d_dM, (void *)d_dL, (void *)d_bptr, (void *)d_bidx,
                        (void *)d_boff, (void *)d_bmat})
            cudaFree(p);
    }
};

// the non-blocking solve (nkb_cg_begin / nkb_cg_poll / nkb_cg_end)
enum SolvePhase
{
    kIdle = 0,  // no solve
    kRun64,     // FP64 CG: blocks of check_interval iterations
    kMixStart,  // mixed: waiting for |b|^2 before the FP32 recurrence starts
    kRun32,     // mixed: FP32 iterations until the recurrence pauses
    kUpdate,    // mixed: waiting for the FP64 residual of a reliable update
    kFinishing, // solution written back, waiting for the last copies
    kFinished   // result ready for nkb_cg_end
};

struct SolveCtx
{
    int phase = kIdle;
    nkb_cg_opts o{};
    cudaStream_t s = nullptr;
    int flags       = 0;
    double *x_user  = nullptr; // caller's x_loc
    double *dx      = nullptr; // device local x (caller's or staging)
    bool use_graph  = false;
    int passes = 0, max_passes = 0, updates = 0, max_upd = 0;
    int restarts = 0, iter_base = 0; // FP32 restarts and the iterations before the last one
    double cycle_min = 0.0;          // smallest iterated FP32 residual of this cycle
    int stall = 0;                   // polls without a new minimum
    bool force_restart = false;
    double thr_final = 0.0, delta = 0.0;
    CGState last32{};
};
} // namespace nkb

using namespace nkb;

struct nkb_sys
{
    std::shared_ptr<SysShared> sh;
    int device = 0;
    cudaStream_t stream = nullptr;
    // read-only views of the shared data
    std::vector<nkb_op *> ops, ops32;
    std::vector<long> off;
    long nloc = 0;
    int nglob = 0, ndir = 0, nn = 0;
    int *d_map = nullptr, *d_aptr = nullptr, *d_aidx = nullptr;
    double *d_sign = nullptr;
    // per instance
    bool has_lambda = false; // lambda overrides the operators' own
    double lambda   = 1.0;
    double *d_dinv  = nullptr;
    double *w = nullptr, *s = nullptr, *x = nullptr, *p = nullptr, *r = nullptr, *q = nullptr;
    double *bglob = nullptr, *yl = nullptr, *tl = nullptr;
    double *partA = nullptr, *partB = nullptr;
    double *partC = nullptr; // block preconditioner partials (2 per CTA)
    int nbC       = 0;
    CGState *st = nullptr;
    CGState *h_st = nullptr; // pinned [3]: FP64 state, FP32 state, state to write
    cudaGraphExec_t graph = nullptr;
    int graph_k = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evq = nullptr;
    double *stage = nullptr; // host-pointer staging (2*nloc)
    long launches = 0;       // kernels launched by the current solve
    float *w32 = nullptr, *s32 = nullptr, *x32 = nullptr, *p32 = nullptr, *r32 = nullptr,
          *q32 = nullptr, *yl32 = nullptr, *dinv32 = nullptr;
    CGState *st32 = nullptr;
    cudaGraphExec_t graph32 = nullptr;
    int graph32_k = 0;
    size_t bytes = 0; // device bytes of this instance
    SolveCtx sv;
};

namespace nkb
{

static const double *LambdaOf(const nkb_sys *S)
{
    return S->has_lambda ? &S->lambda : nullptr;
}

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
                                  S->d_sign ? S->d_sign + o : nullptr, s, skip, LambdaOf(S));
        else
            rc = LaunchOp<double>(op, xin + o, yl + o, nullptr, nullptr, nullptr, nullptr, s, skip,
                                  LambdaOf(S));
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
                                 S->d_sign ? S->d_sign + o : nullptr, s, skip, LambdaOf(S));
        if (rc)
            return rc;
    }
    return NKB_OK;
}

// one FP32 CG iteration (same recurrence as Iteration, FP64 dot sums)
static int Iteration32(nkb_sys *S, cudaStream_t s)
{
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    S->launches += 3 + long(S->ops32.size());
    k_update<float><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st32, S->p32, S->q32, S->x32,
                                                S->r32, S->w32, S->s32, S->dinv32, S->partA, S->nn, 0);
    int rc = Matvec32(S, S->w32, S->yl32, s, &S->st32->done);
    if (rc)
        return rc;
    k_assemble<float><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                  S->d_sign, S->yl32, S->s32, S->w32, S->st32,
                                                  S->partB, S->nn);
    k_scalars<<<1, 1024, 0, s>>>(S->st32, S->partA, nbU, S->partB, nbA, 2);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

// the block step after the diagonal one (k_update / k_precon)
static void BlockPrecon(nkb_sys *S, cudaStream_t s)
{
    const SysShared &h = *S->sh;
    if (!h.nblk)
        return;
    k_block_precon<<<S->nbC, kRedThreads, 0, s>>>(h.nblk, S->ndir, S->st, h.d_bptr, h.d_bidx,
                                                  h.d_boff, h.d_bmat, S->r, S->w, S->partC);
    ++S->launches;
}

static int BlockGrid(int nblk)
{
    return std::max(1, std::min((nblk + kBlockWarps - 1) / kBlockWarps, kBlockGridMax));
}

// kernels of one FP64 iteration
static long IterationLaunches(const nkb_sys *S)
{
    return 3 + long(S->ops.size()) + (S->sh->nblk ? 1 : 0);
}

static int Iteration(nkb_sys *S, cudaStream_t s)
{
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    S->launches += 3 + long(S->ops.size());
    k_update<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->p, S->q, S->x, S->r,
                                                 S->w, S->s, S->d_dinv, S->partA, S->nn, S->sh->nblk ? 0 : 1);
    BlockPrecon(S, s);
    int rc = Matvec(S, S->w, S->yl, true, s, &S->st->done);
    if (rc)
        return rc;
    k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                   S->d_sign, S->yl, S->s, S->w, S->st, S->partB, S->nn);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbU, S->partB, nbA, 2, S->partC, S->nbC);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

// (re)capture K iterations of the FP64 or the FP32 recurrence as a CUDA graph
static int EnsureGraph(nkb_sys *S, bool fp32, cudaStream_t s, int K)
{
    cudaGraphExec_t &ge = fp32 ? S->graph32 : S->graph;
    int &gk             = fp32 ? S->graph32_k : S->graph_k;
    if (ge && gk == K)
        return NKB_OK;
    if (ge)
        cudaGraphExecDestroy(ge);
    ge = nullptr;
    cudaGraph_t g;
    NKB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int crc = NKB_OK;
    for (int k = 0; k < K && !crc; ++k)
        crc = fp32 ? Iteration32(S, s) : Iteration(S, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    S->launches -= long(K) * (3 + long(fp32 ? S->ops32.size() : S->ops.size())); // captured
    if (crc)
        return crc;
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "CG graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "CG graph instantiate: %s", cudaGetErrorString(ce));
    gk = K;
    return NKB_OK;
}

static void DropGraphs(nkb_sys *S)
{
    if (S->graph)
        cudaGraphExecDestroy(S->graph);
    if (S->graph32)
        cudaGraphExecDestroy(S->graph32);
    S->graph = S->graph32 = nullptr;
    S->graph_k = S->graph32_k = 0;
}

} // namespace nkb

namespace nkb
{
static void ViewShared(nkb_sys *S)
{
    const SysShared &h = *S->sh;
    S->device = h.device;
    S->ops    = h.ops;
    S->ops32  = h.ops32;
    S->off    = h.off;
    S->nloc   = h.nloc;
    S->nglob  = h.nglob;
    S->ndir   = h.ndir;
    S->nn     = h.nn;
    S->d_map  = h.d_map;
    S->d_aptr = h.d_aptr;
    S->d_aidx = h.d_aidx;
    S->d_sign = h.d_sign;
}

// per-instance vectors, state, stream and events
static int AllocInstance(nkb_sys *S)
{
    auto dalloc = [&](void **ptr, size_t bytes) -> bool {
        bytes = std::max<size_t>(bytes, 8);
        if (cudaMalloc(ptr, bytes) != cudaSuccess)
            return false;
        S->bytes += bytes;
        return true;
    };
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&S->ev0) != cudaSuccess || cudaEventCreate(&S->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->evq, cudaEventDisableTiming) != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_sys: stream/event creation failed");
    const long nloc = S->nloc;
    bool ok = dalloc((void **)&S->d_dinv, S->nn * sizeof(double)) &&
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
    if (ok && !S->ops32.empty())
        ok = dalloc((void **)&S->w32, S->nglob * sizeof(float)) &&
             dalloc((void **)&S->s32, S->nglob * sizeof(float)) &&
             dalloc((void **)&S->x32, S->nglob * sizeof(float)) &&
             dalloc((void **)&S->p32, S->nn * sizeof(float)) &&
             dalloc((void **)&S->r32, S->nn * sizeof(float)) &&
             dalloc((void **)&S->q32, S->nn * sizeof(float)) &&
             dalloc((void **)&S->dinv32, S->nn * sizeof(float)) &&
             dalloc((void **)&S->yl32, nloc * sizeof(float)) &&
             dalloc((void **)&S->st32, sizeof(CGState));
    if (ok && S->sh->nblk)
    {
        S->nbC = BlockGrid(S->sh->nblk);
        ok     = dalloc((void **)&S->partC, 2 * size_t(S->nbC) * sizeof(double));
    }
    if (!ok)
        return SetError(NKB_ERR_NOMEM, "nkb_sys: device allocation of the CG vectors failed");
    if (cudaMallocHost(&S->h_st, 3 * sizeof(CGState)) != cudaSuccess)
        return SetError(NKB_ERR_NOMEM, "nkb_sys: pinned state");
    std::memset(S->h_st, 0, 3 * sizeof(CGState));
    return NKB_OK;
}

// mass and Laplacian parts of the assembled diagonal, computed once per
// shared system (PreconditionerDiagonal::DiagonalPreconditionerSum with the
// element diagonals split by lambda)
static int EnsureDiagParts(nkb_sys *S)
{
    SysShared &h = *S->sh;
    std::lock_guard<std::mutex> lock(h.mu);
    if (h.d_dM)
        return NKB_OK;
    double *dM = nullptr, *dL = nullptr;
    if (cudaMalloc(&dM, h.nglob * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dL, h.nglob * sizeof(double)) != cudaSuccess)
    {
        cudaFree(dM);
        return SetError(NKB_ERR_NOMEM, "nkb_sys: split diagonal");
    }
    for (size_t c = 0; c < S->ops.size(); ++c)
    {
        int rc = HelmholtzDiag(S->ops[c], S->tl + S->off[c], S->stream, S->yl + S->off[c]);
        if (rc)
        {
            cudaFree(dM);
            cudaFree(dL);
            return rc;
        }
    }
    k_assemble_diag<<<Blocks(S->nglob), kRedThreads, 0, S->stream>>>(S->nglob, S->d_aptr,
                                                                     S->d_aidx, S->d_sign, S->tl,
                                                                     dM);
    k_assemble_diag<<<Blocks(S->nglob), kRedThreads, 0, S->stream>>>(S->nglob, S->d_aptr,
                                                                     S->d_aidx, S->d_sign, S->yl,
                                                                     dL);
    cudaError_t ce = cudaStreamSynchronize(S->stream);
    if (ce != cudaSuccess)
    {
        cudaFree(dM);
        cudaFree(dL);
        return SetError(NKB_ERR_CUDA, "nkb_sys: split diagonal: %s", cudaGetErrorString(ce));
    }
    h.d_dM = dM;
    h.d_dL = dL;
    h.bytes += 2 * h.nglob * sizeof(double);
    return NKB_OK;
}

static bool Busy(const nkb_sys *S)
{
    return S->sv.phase != kIdle;
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
        if (!op || (op->optype != NKB_HELMHOLTZ && op->optype != NKB_DENSE_BLOCK) ||
            op->precision != NKB_FP64 || (op->optype == NKB_DENSE_BLOCK && op->nc != op->nt))
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
    if (desc->ops32)
        for (int c = 0; c < desc->nops; ++c)
        {
            const nkb_op *a = desc->ops[c], *b = desc->ops32[c];
            if (!b || b->optype != NKB_HELMHOLTZ || b->precision != NKB_FP32 ||
                b->nelmt != a->nelmt || b->nc != a->nc)
                return SetError(NKB_ERR_INVALID,
                                "nkb_sys_create: ops32[%d] is not an FP32 twin of ops[%d]", c, c);
        }
    NKB_CUDA_TRY(cudaSetDevice(desc->device));

    auto sh    = std::make_shared<SysShared>();
    sh->device = desc->device;
    sh->nloc   = nloc;
    sh->nglob  = desc->nglob;
    sh->ndir   = desc->ndir;
    sh->nn     = desc->nglob - desc->ndir;
    long o     = 0;
    for (int c = 0; c < desc->nops; ++c)
    {
        sh->ops.push_back(desc->ops[c]);
        if (desc->ops32)
            sh->ops32.push_back(desc->ops32[c]);
        sh->off.push_back(o);
        o += long(desc->ops[c]->nelmt) * desc->ops[c]->nc;
    }
    // global -> local CSR for the deterministic assemble
    std::vector<int> aptr(sh->nglob + 1, 0), aidx(nloc);
    for (long i = 0; i < nloc; ++i)
        aptr[desc->map[i] + 1]++;
    for (int g = 0; g < sh->nglob; ++g)
        aptr[g + 1] += aptr[g];
    {
        std::vector<int> fill(aptr.begin(), aptr.end() - 1);
        for (long i = 0; i < nloc; ++i)
            aidx[fill[desc->map[i]]++] = int(i);
    }
    auto salloc = [&](void **ptr, size_t bytes) -> bool {
        bytes = std::max<size_t>(bytes, 8);
        if (cudaMalloc(ptr, bytes) != cudaSuccess)
            return false;
        sh->bytes += bytes;
        return true;
    };
    if (!salloc((void **)&sh->d_map, nloc * sizeof(int)) ||
        !salloc((void **)&sh->d_aptr, (sh->nglob + 1) * sizeof(int)) ||
        !salloc((void **)&sh->d_aidx, nloc * sizeof(int)) ||
        (desc->sign && !salloc((void **)&sh->d_sign, nloc * sizeof(double))))
        return SetError(NKB_ERR_NOMEM, "nkb_sys_create: device allocation of the map failed");
    NKB_CUDA_TRY(cudaMemcpy(sh->d_map, desc->map, nloc * sizeof(int), cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaMemcpy(sh->d_aptr, aptr.data(), (sh->nglob + 1) * sizeof(int),
                            cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaMemcpy(sh->d_aidx, aidx.data(), nloc * sizeof(int), cudaMemcpyHostToDevice));
    if (desc->sign)
        NKB_CUDA_TRY(cudaMemcpy(sh->d_sign, desc->sign, nloc * sizeof(double),
                                cudaMemcpyHostToDevice));

    nkb_sys *S = new nkb_sys();
    S->sh      = sh;
    ViewShared(S);
    auto fail = [&](int code) {
        nkb_sys_destroy(S);
        return code;
    };
    int rc = AllocInstance(S);
    if (rc)
        return fail(rc);
    // the Hex kernels' variant for gathered launches, timed with this map
    NKB_CUDA_TRY(cudaMemsetAsync(S->w, 0, S->nglob * sizeof(double), S->stream));
    if (S->w32)
        NKB_CUDA_TRY(cudaMemsetAsync(S->w32, 0, S->nglob * sizeof(float), S->stream));
    for (size_t c = 0; c < S->ops.size(); ++c)
    {
        const int *mp = S->d_map + S->off[c];
        const double *sg = S->d_sign ? S->d_sign + S->off[c] : nullptr;
        if ((rc = TuneHexGather(S->ops[c], S->w, S->yl + S->off[c], mp, sg, S->stream)))
            return fail(rc);
        if (!S->ops32.empty() &&
            (rc = TuneHexGather(S->ops32[c], S->w32, S->yl32 + S->off[c], mp, sg, S->stream)))
            return fail(rc);
    }
    // Jacobi diagonal: element diagonals, assembled (modes of sign 0 left
    // out), inverted (PreconditionerDiagonal.cpp:93-125). With one lambda for all operators
    // the mass and Laplacian parts are kept apart (clones with another lambda
    // then only recombine them); otherwise each operator's own lambda.
    bool one_lambda = true;
    for (const nkb_op *op : S->ops)
        one_lambda = one_lambda && op->lambda == S->ops[0]->lambda;
    if (one_lambda)
    {
        if ((rc = EnsureDiagParts(S)))
            return fail(rc);
        k_combine_dinv<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(
            S->nn, S->ndir, S->ops[0]->lambda, sh->d_dM, sh->d_dL, S->d_dinv, S->dinv32);
    }
    else
    {
        for (size_t c = 0; c < S->ops.size(); ++c)
            if ((rc = HelmholtzDiag(S->ops[c], S->tl + S->off[c], S->stream)))
                return fail(rc);
        k_assemble_diag<<<Blocks(S->nglob), kRedThreads, 0, S->stream>>>(
            S->nglob, S->d_aptr, S->d_aidx, S->d_sign, S->tl, S->bglob);
        k_invert<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(S->nn, S->ndir, S->bglob, S->d_dinv);
        if (S->dinv32)
            k_float_copy<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(S->nn, S->d_dinv,
                                                                       S->dinv32);
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(S->stream) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_sys_create: Jacobi diagonal"));
    *out = S;
    return NKB_OK;
}

extern "C" int nkb_sys_clone(const nkb_sys *S, nkb_sys **out)
{
    ClearError();
    if (!S || !out)
        return SetError(NKB_ERR_INVALID, "nkb_sys_clone: NULL argument");
    *out = nullptr;
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    nkb_sys *C = new nkb_sys();
    C->sh      = S->sh;
    ViewShared(C);
    int rc = AllocInstance(C);
    if (rc == NKB_OK)
    {
        C->has_lambda = S->has_lambda;
        C->lambda     = S->lambda;
        if (cudaMemcpyAsync(C->d_dinv, S->d_dinv, S->nn * sizeof(double), cudaMemcpyDeviceToDevice,
                            C->stream) != cudaSuccess ||
            (C->dinv32 && cudaMemcpyAsync(C->dinv32, S->dinv32, S->nn * sizeof(float),
                                          cudaMemcpyDeviceToDevice, C->stream) != cudaSuccess) ||
            cudaStreamSynchronize(C->stream) != cudaSuccess)
            rc = SetError(NKB_ERR_CUDA, "nkb_sys_clone: copy of the Jacobi diagonal");
    }
    if (rc)
    {
        nkb_sys_destroy(C);
        return rc;
    }
    *out = C;
    return NKB_OK;
}

extern "C" int nkb_sys_set_lambda(nkb_sys *S, double lambda)
{
    ClearError();
    if (!S || !std::isfinite(lambda))
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_lambda: bad arguments");
    if (Busy(S))
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_lambda: a solve is in progress");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    int rc = EnsureDiagParts(S);
    if (rc)
        return rc;
    k_combine_dinv<<<Blocks(S->nn), kRedThreads, 0, S->stream>>>(
        S->nn, S->ndir, lambda, S->sh->d_dM, S->sh->d_dL, S->d_dinv, S->dinv32);
    NKB_CUDA_TRY(cudaGetLastError());
    NKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    S->lambda     = lambda;
    S->has_lambda = true;
    DropGraphs(S); // the captured launches carry the old lambda
    return NKB_OK;
}

extern "C" int nkb_sys_set_blocks(nkb_sys *S, int nblk, const int *bptr, const int *bidx,
                                  const double *binv)
{
    ClearError();
    if (!S || nblk < 1 || !bptr || !bidx || !binv)
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: bad arguments");
    if (Busy(S))
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: a solve is in progress");
    SysShared &h = *S->sh;
    if (S->sh.use_count() > 1)
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: set the blocks before cloning");
    if (h.nblk)
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: blocks already set");
    if (h.grouped)
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_sys_set_blocks: a shard of a sharded group");
    if (bptr[0] != 0)
        return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: bptr[0] = %d", bptr[0]);
    std::vector<long> boff(nblk);
    std::vector<char> seen(S->nn, 0);
    long tot = 0;
    for (int b = 0; b < nblk; ++b)
    {
        const int n = bptr[b + 1] - bptr[b];
        if (n < 1 || n > kBlockMax)
            return SetError(NKB_ERR_INVALID, "nkb_sys_set_blocks: block %d has %d rows (1..%d)", b,
                            n, kBlockMax);
        for (int j = bptr[b]; j < bptr[b + 1]; ++j)
        {
            if (bidx[j] < 0 || bidx[j] >= S->nn || seen[bidx[j]])
                return SetError(NKB_ERR_INVALID,
                                "nkb_sys_set_blocks: index %d of block %d outside [0,%d) or "
                                "in two blocks",
                                bidx[j], b, S->nn);
            seen[bidx[j]] = 1;
        }
        boff[b] = tot;
        tot += long(n) * n;
    }
    const long nidx = bptr[nblk];
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    int *dp = nullptr, *di = nullptr;
    long *dof = nullptr;
    double *dm = nullptr;
    auto release = [&]() {
        cudaFree(dp);
        cudaFree(di);
        cudaFree(dof);
        cudaFree(dm);
    };
    if (cudaMalloc(&dp, (nblk + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&di, nidx * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dof, nblk * sizeof(long)) != cudaSuccess ||
        cudaMalloc(&dm, tot * sizeof(double)) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_sys_set_blocks: %ld doubles of blocks", tot);
    }
    if (cudaMemcpy(dp, bptr, (nblk + 1) * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(di, bidx, nidx * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dof, boff.data(), nblk * sizeof(long), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dm, binv, tot * sizeof(double), cudaMemcpyDefault) != cudaSuccess ||
        cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) // binv may be device memory
    {
        release();
        return SetError(NKB_ERR_CUDA, "nkb_sys_set_blocks: upload");
    }
    double *pc   = nullptr;
    const int nc = BlockGrid(nblk);
    if (cudaMalloc(&pc, 2 * size_t(nc) * sizeof(double)) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_sys_set_blocks: partials");
    }
    S->partC = pc;
    S->nbC   = nc;
    S->bytes += 2 * size_t(nc) * sizeof(double);
    h.d_bptr = dp;
    h.d_bidx = di;
    h.d_boff = dof;
    h.d_bmat = dm;
    h.nblk   = nblk;
    h.bytes += (nblk + 1) * sizeof(int) + nidx * sizeof(int) + nblk * sizeof(long) +
               tot * sizeof(double);
    DropGraphs(S); // graphs captured so far lack the block step
    return NKB_OK;
}

extern "C" int nkb_sys_footprint(const nkb_sys *S, size_t *shared_bytes, size_t *instance_bytes)
{
    ClearError();
    if (!S)
        return SetError(NKB_ERR_INVALID, "nkb_sys_footprint: NULL system");
    if (shared_bytes)
        *shared_bytes = S->sh->bytes;
    if (instance_bytes)
        *instance_bytes = S->bytes;
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
        S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, loc, glob, nullptr, nullptr, nullptr, S->nn);
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
// The solve runs as a sequence of device work blocks; after each block the
// relevant CG state is copied to pinned host memory and an event recorded.
// nkb_cg_poll looks at that state once the event has completed and issues the
// next block, so several systems can be driven concurrently from one host
// thread (each on its own stream) and nkb_cg_solve is the same machine
// polled with waits.

static int QueueState(nkb_sys *S, int which)
{
    const CGState *src = which == 0 ? S->st : S->st32;
    NKB_CUDA_TRY(cudaMemcpyAsync(S->h_st + which, src, sizeof(CGState), cudaMemcpyDeviceToHost,
                                 S->sv.s));
    NKB_CUDA_TRY(cudaEventRecord(S->evq, S->sv.s));
    return NKB_OK;
}

// h0 -> S->st: a fresh state with the stopping rule (NekLinSysIter.cpp:57)
static int ResetState(nkb_sys *S)
{
    CGState &h0 = S->h_st[2];
    std::memset(&h0, 0, sizeof(h0));
    const double tol = std::fmax(S->sv.o.tol, 1.0e-16);
    h0.tol2          = tol * tol;
    h0.maxit         = S->sv.o.maxit;
    NKB_CUDA_TRY(cudaMemcpyAsync(S->st, &h0, sizeof(h0), cudaMemcpyHostToDevice, S->sv.s));
    return NKB_OK;
}

// x_loc += GlobalToLocal(x) (the Dirichlet part of x is zero), copies back;
// `fin` (if given) replaces the device state first
static int Finish(nkb_sys *S, const CGState *fin)
{
    SolveCtx &v    = S->sv;
    cudaStream_t s = v.s;
    if (fin)
    {
        S->h_st[2] = *fin;
        NKB_CUDA_TRY(cudaMemcpyAsync(S->st, S->h_st + 2, sizeof(CGState), cudaMemcpyHostToDevice, s));
    }
    k_global_to_local<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, S->d_map, S->d_sign, S->x,
                                                               S->tl);
    k_axpy_loc<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, 1.0, S->tl, v.dx);
    S->launches += 2;
    NKB_CUDA_TRY(cudaEventRecord(S->ev1, s));
    if (v.flags & NKB_HOST_PTRS)
        NKB_CUDA_TRY(cudaMemcpyAsync(v.x_user, v.dx, S->nloc * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
    v.phase = kFinishing;
    return QueueState(S, 0);
}

static int Begin64(nkb_sys *S)
{
    SolveCtx &v    = S->sv;
    cudaStream_t s = v.s;
    int rc         = ResetState(S);
    if (rc)
        return rc;
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    k_init<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->bglob, S->r, S->x, S->w, S->s, S->p,
                                       S->q, S->partA, nullptr, S->nn);
    // partA holds (b,b) in [0] and (r,r) in [1]; k_scalars mode 0 reads eps
    // from partA[1] and rhs from partB[0]
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbA, S->partA, nbA, 0);
    k_precon<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->r, S->w, S->d_dinv,
                                                 S->partA, S->nn);
    BlockPrecon(S, s);
    if ((rc = Matvec(S, S->w, S->yl, true, s)))
        return rc;
    k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                   S->d_sign, S->yl, S->s, S->w, S->st, S->partB, S->nn);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbU, S->partB, nbA, 1, S->partC, S->nbC);
    NKB_CUDA_TRY(cudaGetLastError());
    S->launches += 5 + long(S->ops.size());
    v.use_graph = v.o.use_graph != 0 && s != cudaStreamLegacy && s != cudaStreamPerThread;
    if (v.use_graph && (rc = EnsureGraph(S, false, s, v.o.check_interval)))
        return rc;
    v.passes     = 0;
    v.max_passes = v.o.maxit / v.o.check_interval + 2;
    v.phase      = kRun64;
    return QueueState(S, 0);
}

static int Step64(nkb_sys *S)
{
    SolveCtx &v = S->sv;
    if (S->h_st[0].done || v.passes >= v.max_passes)
        return Finish(S, nullptr);
    const int K = v.o.check_interval;
    if (v.use_graph)
    {
        NKB_CUDA_TRY(cudaGraphLaunch(S->graph, v.s));
        S->launches += long(K) * IterationLaunches(S);
    }
    else
    {
        for (int k = 0; k < K; ++k)
        {
            int rc = Iteration(S, v.s);
            if (rc)
                return rc;
        }
    }
    ++v.passes;
    return QueueState(S, 0);
}

// Mixed precision: FP32 PCG (operators, vectors, preconditioner in FP32; dot
// products summed in FP64) with reliable updates. Whenever the iterated FP32
// residual has dropped by the factor delta since the last update, the FP32
// correction is folded into the FP64 solution, the true residual b - A x is
// recomputed with the FP64 operators, and the FP32 recurrence continues from
// it with its search direction kept (no restart, so the Krylov convergence is
// preserved). Convergence is decided on the FP64 residual only, with the
// FP64 criterion eps < tol^2 |b|^2.
// The FP32 operator's rounding is relative to |A||p|, not |Ap|: on smooth
// vectors it grows with the condition number, and the true residual can then
// drift far from the iterated one (the search directions are no longer
// conjugate). When an update finds |r_true|^2 > kDrift |r_iter|^2 the FP32
// recurrence restarts from the true residual (iterative refinement) and runs
// each restarted cycle to the deeper reduction kRestartReduction.
// The recurrence can also stall (the iterated residual stops falling): after
// kStallPolls polls without a new minimum (10 % lower) the cycle is ended by a
// reliable update and a restart.
constexpr double kDrift            = 2.0;
constexpr double kRestartReduction = 1.0e-3;
constexpr int kStallPolls          = 8;

static int BeginMixed(nkb_sys *S)
{
    SolveCtx &v    = S->sv;
    cudaStream_t s = v.s;
    if (s == cudaStreamLegacy || s == cudaStreamPerThread)
        return SetError(NKB_ERR_INVALID, "mixed-precision solve needs a created stream");
    int rc = ResetState(S);
    if (rc)
        return rc;
    const int nbA = Blocks(S->nglob);
    k_init<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->bglob, S->r, S->x, S->w, S->s, S->p,
                                       S->q, S->partA, nullptr, S->nn);
    k_scalars<<<1, 1024, 0, s>>>(S->st, S->partA, nbA, S->partA, nbA, 0);
    S->launches += 2;
    if ((rc = EnsureGraph(S, true, s, v.o.check_interval)))
        return rc;
    v.delta      = v.o.inner_tol > 0 ? std::fmin(v.o.inner_tol, 0.5) : 0.1;
    v.max_upd    = v.o.max_outer > 0 ? v.o.max_outer : 1000;
    v.updates    = 0;
    v.passes     = 0;
    v.max_passes = v.o.maxit / v.o.check_interval + 2;
    v.phase      = kMixStart;
    return QueueState(S, 0);
}

// FP32 recurrence from r32 (reset: x32 = 0 and a first direction; otherwise
// a continuation after a reliable update)
static int Launch32Start(nkb_sys *S, double eps, bool reset, double reduction)
{
    SolveCtx &v    = S->sv;
    cudaStream_t s = v.s;
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    if (reset)
        k_init_inner<<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->r, S->r32, S->x32, S->w32,
                                                 S->s32, S->p32, S->q32, S->partA);
    k_resume<<<1, 1, 0, s>>>(S->st32, std::fmax(reduction * reduction * eps, v.thr_final),
                             std::max(v.o.maxit - v.iter_base, 1), reset ? 1 : 0);
    k_precon<float><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st32, S->r32, S->w32, S->dinv32,
                                                S->partA, S->nn);
    int rc = Matvec32(S, S->w32, S->yl32, s, &S->st32->done);
    if (rc)
        return rc;
    k_assemble<float><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                  S->d_sign, S->yl32, S->s32, S->w32, S->st32,
                                                  S->partB, S->nn);
    k_scalars<<<1, 1024, 0, s>>>(S->st32, S->partA, nbU, S->partB, nbA, reset ? 1 : 3);
    NKB_CUDA_TRY(cudaGetLastError());
    S->launches += (reset ? 5 : 4) + long(S->ops32.size());
    v.phase     = kRun32;
    v.cycle_min = eps;
    v.stall     = 0;
    return QueueState(S, 1);
}

static int StepMixStart(nkb_sys *S)
{
    SolveCtx &v     = S->sv;
    const CGState h = S->h_st[0];
    v.thr_final     = h.tol2 * h.rhs_mag;
    if (h.done)
        return Finish(S, nullptr);
    return Launch32Start(S, h.eps, true, v.delta);
}

static int StepRun32(nkb_sys *S)
{
    SolveCtx &v       = S->sv;
    const CGState h32 = S->h_st[1];
    if (!h32.done)
    {
        if (h32.eps < 0.9 * v.cycle_min)
        {
            v.cycle_min = h32.eps;
            v.stall     = 0;
        }
        else if (++v.stall >= kStallPolls)
        {
            v.force_restart = true;
        }
    }
    if (!h32.done && !v.force_restart && v.passes < v.max_passes)
    {
        NKB_CUDA_TRY(cudaGraphLaunch(S->graph32, v.s));
        S->launches += long(v.o.check_interval) * (3 + long(S->ops32.size()));
        ++v.passes;
        return QueueState(S, 1);
    }
    v.last32 = h32;
    if (h32.status == NKB_ERR_NONFINITE)
    {
        CGState fin = S->h_st[0];
        fin.done    = 1;
        fin.status  = NKB_ERR_NONFINITE;
        fin.iter    = v.iter_base + h32.iter;
        return Finish(S, &fin);
    }
    // reliable update: x += x32 (x32 = 0), r = b - A x in FP64, r32 = (float) r
    cudaStream_t s = v.s;
    const int nbU = Blocks(S->nn), nbA = Blocks(S->nglob);
    k_add_correction<<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->x, S->x32);
    int rc = Matvec(S, S->x, S->yl, true, s);
    if (rc)
        return rc;
    k_assemble<double><<<nbA, kRedThreads, 0, s>>>(S->nglob, S->ndir, S->d_aptr, S->d_aidx,
                                                   S->d_sign, S->yl, S->s, nullptr, nullptr,
                                                   nullptr, S->nn);
    k_residual<<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->bglob, S->s, S->r, S->r32, S->partA);
    k_scalars_outer<<<1, 1024, 0, s>>>(S->st, S->partA, nbU);
    NKB_CUDA_TRY(cudaGetLastError());
    S->launches += 4 + long(S->ops.size());
    ++v.updates;
    v.phase = kUpdate;
    return QueueState(S, 0);
}

static int StepUpdate(nkb_sys *S)
{
    SolveCtx &v = S->sv;
    CGState h   = S->h_st[0];
    bool stop   = true;
    int status  = NKB_OK;
    if (!std::isfinite(h.eps))
        status = NKB_ERR_NONFINITE;
    else if (h.eps < v.thr_final)
        status = NKB_OK;
    else if (v.last32.status == NKB_ERR_NOT_CONVERGED || v.updates >= v.max_upd ||
             v.iter_base + v.last32.iter >= v.o.maxit ||
             v.passes >= v.max_passes)
        status = NKB_ERR_NOT_CONVERGED;
    else
        stop = false;
    if (stop)
    {
        h.done   = 1;
        h.status = status;
        h.iter   = v.iter_base + v.last32.iter;
        return Finish(S, &h);
    }
    if (v.force_restart || h.eps > kDrift * v.last32.eps)
    {
        v.force_restart = false;
        // the FP32 recurrence has lost track of the true residual: restart it
        v.iter_base += v.last32.iter;
        ++v.restarts;
        return Launch32Start(S, h.eps, true, kRestartReduction);
    }
    return Launch32Start(S, h.eps, false, v.delta);
}
} // namespace nkb

extern "C" int nkb_cg_begin(nkb_sys *S, const double *b_loc, double *x_loc,
                            const nkb_cg_opts *opts, int flags, void *stream)
{
    ClearError();
    if (!S || !b_loc || !x_loc)
        return SetError(NKB_ERR_INVALID, "nkb_cg_begin: NULL argument");
    if (Busy(S))
        return SetError(NKB_ERR_INVALID, "nkb_cg_begin: a solve is already in progress");
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
        return SetError(NKB_ERR_INVALID, "nkb_cg_begin: mixed precision needs FP32 operators "
                                         "(nkb_sys_desc.ops32)");
    if (o.mixed && S->sh->nblk)
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_cg_begin: the block preconditioner is FP64 only");
    if (S->sh->grouped)
        return SetError(NKB_ERR_INVALID, "nkb_cg_begin: a shard of a sharded group solves through "
                                         "nkb_shard_group_solve");
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    SolveCtx &v = S->sv;
    v           = SolveCtx();
    v.o         = o;
    v.flags     = flags;
    // NULL (or the legacy default stream) -> the system's own stream
    v.s              = stream ? static_cast<cudaStream_t>(stream) : S->stream;
    cudaStream_t s   = v.s;
    const long nloc  = S->nloc;
    const double *db = b_loc;
    v.x_user         = x_loc;
    v.dx             = x_loc;
    if (flags & NKB_HOST_PTRS)
    {
        if (!S->stage)
        {
            if (cudaMalloc(&S->stage, 2 * nloc * sizeof(double)) != cudaSuccess)
                return SetError(NKB_ERR_NOMEM, "nkb_cg_begin: staging buffers");
            S->bytes += 2 * nloc * sizeof(double);
        }
        NKB_CUDA_TRY(cudaMemcpyAsync(S->stage, b_loc, nloc * sizeof(double), cudaMemcpyHostToDevice, s));
        NKB_CUDA_TRY(cudaMemcpyAsync(S->stage + nloc, x_loc, nloc * sizeof(double),
                                     cudaMemcpyHostToDevice, s));
        db   = S->stage;
        v.dx = S->stage + nloc;
    }
    NKB_CUDA_TRY(cudaEventRecord(S->ev0, s));
    S->launches = 0;
    // Dirichlet lifting (GlobalLinSysIterativeFull.cpp:104-164):
    // rhs = b - A x_D (local), gloIn = Assemble(rhs)
    int rc = Matvec(S, v.dx, S->yl, false, s);
    if (rc == NKB_OK)
    {
        k_sub_loc<<<Blocks(nloc), kRedThreads, 0, s>>>(nloc, db, S->yl, S->tl);
        k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
            S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, S->tl, S->bglob, nullptr, nullptr,
            nullptr, S->nn);
        S->launches += 2 + long(S->ops.size());
        rc = o.mixed ? BeginMixed(S) : Begin64(S);
    }
    if (rc)
        v.phase = kIdle;
    return rc;
}

extern "C" int nkb_cg_poll(nkb_sys *S, int wait, int *done)
{
    ClearError();
    if (!S || !done)
        return SetError(NKB_ERR_INVALID, "nkb_cg_poll: NULL argument");
    *done       = 0;
    SolveCtx &v = S->sv;
    if (v.phase == kIdle)
        return SetError(NKB_ERR_INVALID, "nkb_cg_poll: no solve in progress");
    if (v.phase == kFinished)
    {
        *done = 1;
        return NKB_OK;
    }
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    if (wait)
    {
        const cudaError_t e = cudaEventSynchronize(S->evq);
        if (e != cudaSuccess)
        {
            v.phase = kIdle;
            return SetError(NKB_ERR_CUDA, "nkb_cg_poll: %s", cudaGetErrorString(e));
        }
    }
    else
    {
        const cudaError_t q = cudaEventQuery(S->evq);
        if (q == cudaErrorNotReady)
            return NKB_OK;
        if (q != cudaSuccess)
        {
            v.phase = kIdle;
            return SetError(NKB_ERR_CUDA, "nkb_cg_poll: %s", cudaGetErrorString(q));
        }
    }
    int rc = NKB_OK;
    switch (v.phase)
    {
        case kRun64: rc = Step64(S); break;
        case kMixStart: rc = StepMixStart(S); break;
        case kRun32: rc = StepRun32(S); break;
        case kUpdate: rc = StepUpdate(S); break;
        case kFinishing:
            v.phase = kFinished;
            *done   = 1;
            break;
        default: break;
    }
    if (rc)
        v.phase = kIdle;
    return rc;
}

extern "C" int nkb_cg_end(nkb_sys *S, nkb_cg_report *rep)
{
    ClearError();
    if (!S)
        return SetError(NKB_ERR_INVALID, "nkb_cg_end: NULL system");
    SolveCtx &v = S->sv;
    if (v.phase != kFinished)
        return SetError(NKB_ERR_INVALID, "nkb_cg_end: the solve has not finished (poll until done)");
    v.phase         = kIdle;
    const CGState h = S->h_st[0];
    if (rep)
    {
        rep->iterations       = h.iter;
        rep->outer_iterations = v.updates;
        rep->rel_residual     = std::sqrt(h.eps / h.rhs_mag);
        rep->converged        = (h.done && h.status == NKB_OK) ? 1 : 0;
        float ms              = 0.f;
        cudaEventElapsedTime(&ms, S->ev0, S->ev1);
        rep->device_ms       = ms;
        rep->kernel_launches = S->launches;
        rep->restarts        = v.restarts;
    }
    // a bounded wait that gave up inside an operator kernel left some
    // element outputs unwritten: the solve's result cannot be trusted
    NKB_CUDA_TRY(cudaSetDevice(S->device));
    for (const auto *ops : {&S->ops, &S->ops32})
        for (nkb_op *op : *ops)
            if (int rc = CheckOpError(op))
                return rc;
    if (h.status == NKB_ERR_NONFINITE)
        return SetError(NKB_ERR_NONFINITE, "nkb_cg_solve: non-finite CG scalar at iteration %d", h.iter);
    if (h.status == NKB_ERR_NOT_CONVERGED || !h.done)
        return SetError(NKB_ERR_NOT_CONVERGED,
                        "nkb_cg_solve: CG iterations made = %d exceeded maxit (error = %g)", h.iter,
                        std::sqrt(h.eps / h.rhs_mag));
    return NKB_OK;
}

extern "C" int nkb_cg_solve(nkb_sys *S, const double *b_loc, double *x_loc,
                            const nkb_cg_opts *opts, nkb_cg_report *rep, int flags, void *stream)
{
    int rc = nkb_cg_begin(S, b_loc, x_loc, opts, flags, stream);
    if (rc)
        return rc;
    int done = 0;
    while (!done)
        if ((rc = nkb_cg_poll(S, 1, &done)))
            return rc;
    return nkb_cg_end(S, rep);
}

extern "C" int nkb_sys_profile_iteration(nkb_sys *S, int iters, nkb_sys_profile *prof)
{
    ClearError();
    if (!S || !prof || iters < 1)
        return SetError(NKB_ERR_INVALID, "nkb_sys_profile_iteration: bad arguments");
    if (Busy(S))
        return SetError(NKB_ERR_INVALID, "nkb_sys_profile_iteration: a solve is in progress");
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
                                                       S->partB, S->nn);
    NKB_CUDA_TRY(cudaEventRecord(e[2], s));
    // the update kernel with alpha = beta = 0 leaves x unchanged and w = dinv r
    CGState zero = run;
    zero.alpha = zero.beta = 0.0;
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    NKB_CUDA_TRY(cudaMemcpy(S->st, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    NKB_CUDA_TRY(cudaEventRecord(e[2], s));
    for (int it = 0; it < iters; ++it)
        k_update<double><<<nbU, kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->p, S->q, S->x,
                                                     S->r, S->w, S->s, S->d_dinv, S->partA, S->nn, S->sh->nblk ? 0 : 1);
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
    if (S->stream)
        cudaStreamSynchronize(S->stream); // a solve may still be in flight
    if (S->sv.s && S->sv.s != S->stream)
        cudaStreamSynchronize(S->sv.s);
    DropGraphs(S);
    for (void *ptr : {(void *)S->w32, (void *)S->s32, (void *)S->x32, (void *)S->p32,
                      (void *)S->r32, (void *)S->q32, (void *)S->dinv32, (void *)S->yl32,
                      (void *)S->st32, (void *)S->d_dinv, (void *)S->w, (void *)S->s,
                      (void *)S->x, (void *)S->bglob, (void *)S->p, (void *)S->r, (void *)S->q,
                      (void *)S->yl, (void *)S->tl, (void *)S->partA, (void *)S->partB,
                      (void *)S->partC, (void *)S->st, (void *)S->stage})
        cudaFree(ptr);
    if (S->h_st)
        cudaFreeHost(S->h_st);
    for (cudaEvent_t e : {S->ev0, S->ev1, S->evq})
        if (e)
            cudaEventDestroy(e);
    if (S->stream)
        cudaStreamDestroy(S->stream);
    S->sh.reset(); // the shared map and diagonal go with the last user
    delete S;
}

#include "nkb_cg_shard.cuh"
