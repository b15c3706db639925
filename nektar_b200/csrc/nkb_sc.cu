// Static condensation of per-element matrices on the device: the set-up of
// GlobalLinSysIterativeStaticCond (MultiRegions/GlobalLinSysIterativeStaticCond
// .cpp:199, v_AssembleSchurComplement; the maps of GlobalLinSysStaticCond::
// v_Solve, GlobalLinSysStaticCond.cpp:98-227) for element matrices that are
// already on the device (nkb_op_element_matrices with device pointers).
//
// Per element, with the local modes split into boundary modes bm (nb) and
// interior modes im (ni) and K the element matrix (K[i][j] = output i for
// unit input j):
//   Kii = L L^T                         (Cholesky; Kii is SPD for lambda > 0)
//   [X | Xi] = Kii^-1 [Kib | I]         (forward and back substitution)
//   S0 = Kbb - Kbi X                    (the Schur complement)
//   C  = Kbi Xi                         (= Kbi Kii^-1)
// and with a transform R (nb x nb; the low-energy basis, or the identity):
//   S = R S0 R^T
//   W (nb x nc): W[:, bm] = R,   W[:, im] = -R C        b~ = W b_e
//   V (nc x (nb+ni)): V[bm, :nb] = R^T, V[im, :nb] = -X R^T, V[im, nb:] = Xi
//                                        x_e = V [x~_e, b_i,e]
// One CTA per element, all arithmetic FP64 in a fixed order (the result does
// not depend on the launch); elements are processed in chunks through a
// bounded workspace. Elements without interior modes (ni = 0: tetrahedra at
// P <= 3, prisms at P <= 2) give S = R Kbb R^T, W = R, V = R^T.
#include "nkb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace nkb
{
namespace
{
constexpr int kScThreads = 256;
constexpr int kTile      = 32;

// C[M x N] = alpha op(A) op(B) + beta C (row-major with leading dimensions;
// op(A)[i][k] = TA ? A[k * lda + i] : A[i * lda + k], op(B)[k][j] likewise),
// by the whole CTA: 32 x 32 output tiles, 2 x 2 outputs per thread, 32-deep
// K steps staged in shared memory, sums in a fixed order
struct GemmTiles
{
    double a[kTile][kTile + 1], b[kTile][kTile + 1];
};

template <bool TA, bool TB>
__device__ void CtaGemm(GemmTiles &sm, int M, int N, int K, double alpha, const double *A, int lda,
                        const double *B, int ldb, double beta, double *C, int ldc)
{
    auto &sA = sm.a;
    auto &sB = sm.b;
    const int tid = threadIdx.x, tr = tid / 16, tc = tid % 16; // 16 x 16 threads
    for (int i0 = 0; i0 < M; i0 += kTile)
        for (int j0 = 0; j0 < N; j0 += kTile)
        {
            double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
            for (int k0 = 0; k0 < K; k0 += kTile)
            {
                // consecutive threads read consecutive addresses of A and B
                for (int t = tid; t < kTile * kTile; t += kScThreads)
                {
                    const int r = t / kTile, c = t % kTile;
                    {
                        const int ii = TA ? c : r, kk = TA ? r : c;
                        const int ia = i0 + ii, ka = k0 + kk;
                        sA[ii][kk] = (ia < M && ka < K)
                                         ? (TA ? A[long(ka) * lda + ia] : A[long(ia) * lda + ka])
                                         : 0.0;
                    }
                    {
                        const int kk = TB ? c : r, jj = TB ? r : c;
                        const int kb = k0 + kk, jb = j0 + jj;
                        sB[kk][jj] = (kb < K && jb < N)
                                         ? (TB ? B[long(jb) * ldb + kb] : B[long(kb) * ldb + jb])
                                         : 0.0;
                    }
                }
                __syncthreads();
#pragma unroll 8
                for (int k = 0; k < kTile; ++k)
                {
                    const double a0 = sA[2 * tr][k], a1 = sA[2 * tr + 1][k];
                    const double b0 = sB[k][2 * tc], b1 = sB[k][2 * tc + 1];
                    acc[0][0] = fma(a0, b0, acc[0][0]);
                    acc[0][1] = fma(a0, b1, acc[0][1]);
                    acc[1][0] = fma(a1, b0, acc[1][0]);
                    acc[1][1] = fma(a1, b1, acc[1][1]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int v = 0; v < 2; ++v)
                {
                    const int i = i0 + 2 * tr + u, j = j0 + 2 * tc + v;
                    if (i < M && j < N)
                    {
                        double *c = C + long(i) * ldc + j;
                        *c        = beta == 0.0 ? alpha * acc[u][v] : fma(alpha, acc[u][v], beta * *c);
                    }
                }
        }
    __syncthreads();
}

struct ScArgs
{
    int nc, nb, ni;
    const double *K; // [e][nc][nc] of the chunk
    const int *bm, *im;
    const double *R; // nb x nb or null (identity)
    double *S, *W, *V; // outputs of the chunk
    double *ws;        // workspace, wstride doubles per CTA
    long wstride;
    int nelmt; // elements in the chunk
    int *err;
};

__global__ void __launch_bounds__(kScThreads) k_condense(ScArgs a)
{
    const int e = blockIdx.x;
    if (e >= a.nelmt)
        return;
    const int nc = a.nc, nb = a.nb, ni = a.ni, m = nb + ni, tid = threadIdx.x;
    const int nmax = nb > ni ? nb : ni;
    __shared__ GemmTiles tiles;
    const double *Ke = a.K + long(e) * nc * nc;
    double *Kii = a.ws + long(e) * a.wstride; // ni x ni
    double *Z   = Kii + long(ni) * ni;        // ni x m: [Kib | I] -> [X | Xi]
    double *Kbi = Z + long(ni) * m;           // nb x ni, later R S0 (nb x nb)
    double *T1  = Kbi + long(nb) * nmax;      // nb x nmax
    double *T2  = T1 + long(nb) * nmax;       // nmax x nmax
    double *S   = a.S + long(e) * nb * nb;
    double *W   = a.W + long(e) * nb * nc;
    double *V   = a.V + long(e) * nc * m;

    // blocks of K
    for (long t = tid; t < long(ni) * ni; t += kScThreads)
    {
        const int r = int(t / ni), c = int(t % ni);
        Kii[t] = Ke[long(a.im[r]) * nc + a.im[c]];
    }
    for (long t = tid; t < long(ni) * m; t += kScThreads)
    {
        const int r = int(t / m), c = int(t % m);
        Z[t] = c < nb ? Ke[long(a.im[r]) * nc + a.bm[c]] : (c - nb == r ? 1.0 : 0.0);
    }
    for (long t = tid; t < long(nb) * ni; t += kScThreads)
    {
        const int r = int(t / ni), c = int(t % ni);
        Kbi[t] = Ke[long(a.bm[r]) * nc + a.im[c]];
    }
    double *S0 = a.R ? T2 : S; // Kbb, then the Schur complement
    for (long t = tid; t < long(nb) * nb; t += kScThreads)
    {
        const int r = int(t / nb), c = int(t % nb);
        S0[t] = Ke[long(a.bm[r]) * nc + a.bm[c]];
    }
    __syncthreads();

    // Cholesky of Kii in place (lower triangle), right-looking
    __shared__ double piv;
    __shared__ int bad;
    if (tid == 0)
        bad = 0;
    for (int k = 0; k < ni; ++k)
    {
        if (tid == 0)
        {
            const double d = Kii[long(k) * ni + k];
            if (!(d > 0.0))
            {
                bad = 1;
                piv = 1.0;
            }
            else
                piv = sqrt(d);
            Kii[long(k) * ni + k] = piv;
        }
        __syncthreads();
        const double p = piv;
        for (int i = k + 1 + tid; i < ni; i += kScThreads)
            Kii[long(i) * ni + k] /= p;
        __syncthreads();
        const int r = ni - k - 1;
        for (long t = tid; t < long(r) * r; t += kScThreads)
        {
            const int i = k + 1 + int(t / r), j = k + 1 + int(t % r);
            if (j <= i)
                Kii[long(i) * ni + j] = fma(-Kii[long(i) * ni + k], Kii[long(j) * ni + k],
                                            Kii[long(i) * ni + j]);
        }
        __syncthreads();
    }
    if (bad && tid == 0)
        atomicExch(a.err, 1);

    // [X | Xi] = Kii^-1 [Kib | I]: blocked forward then back substitution.
    // Each 32-row diagonal block is solved a column per thread; the rows
    // after it (forward) or before it (back) are updated by one CTA GEMM.
    for (int k0 = 0; k0 < ni; k0 += kTile)
    {
        const int kb = min(kTile, ni - k0);
        for (int c = tid; c < m; c += kScThreads)
            for (int i = k0; i < k0 + kb; ++i)
            {
                double s = Z[long(i) * m + c];
                for (int k = k0; k < i; ++k)
                    s = fma(-Kii[long(i) * ni + k], Z[long(k) * m + c], s);
                Z[long(i) * m + c] = s / Kii[long(i) * ni + i];
            }
        __syncthreads();
        if (k0 + kb < ni) // Z[k0+kb:] -= L[k0+kb:, k0:k0+kb] Z[k0:k0+kb]
            CtaGemm<false, false>(tiles, ni - k0 - kb, m, kb, -1.0, Kii + long(k0 + kb) * ni + k0, ni,
                                  Z + long(k0) * m, m, 1.0, Z + long(k0 + kb) * m, m);
    }
    for (int k0 = ni > 0 ? ((ni - 1) / kTile) * kTile : -1; k0 >= 0; k0 -= kTile)
    {
        const int kb = min(kTile, ni - k0);
        for (int c = tid; c < m; c += kScThreads)
            for (int i = k0 + kb - 1; i >= k0; --i)
            {
                double s = Z[long(i) * m + c];
                for (int k = i + 1; k < k0 + kb; ++k)
                    s = fma(-Kii[long(k) * ni + i], Z[long(k) * m + c], s);
                Z[long(i) * m + c] = s / Kii[long(i) * ni + i];
            }
        __syncthreads();
        if (k0 > 0) // Z[:k0] -= L[k0:k0+kb, :k0]^T Z[k0:k0+kb]
            CtaGemm<true, false>(tiles, k0, m, kb, -1.0, Kii + long(k0) * ni, ni, Z + long(k0) * m, m, 1.0,
                                 Z, m);
    }

    // S0 = Kbb - Kbi X
    CtaGemm<false, false>(tiles, nb, nb, ni, -1.0, Kbi, ni, Z, m, 1.0, S0, nb);
    // C = Kbi Xi (nb x ni) into T1
    CtaGemm<false, false>(tiles, nb, ni, ni, 1.0, Kbi, ni, Z + nb, m, 0.0, T1, ni);
    if (a.R)
    {
        // S = R S0 R^T (T2 holds S0; R S0 into Kbi, whose values are done)
        double *RS0 = Kbi; // the region holds nb x max(nb, ni)
        CtaGemm<false, false>(tiles, nb, nb, nb, 1.0, a.R, nb, S0, nb, 0.0, RS0, nb);
        CtaGemm<false, true>(tiles, nb, nb, nb, 1.0, RS0, nb, a.R, nb, 0.0, S, nb);
        // -R C into T2 (nb x ni)
        CtaGemm<false, false>(tiles, nb, ni, nb, -1.0, a.R, nb, T1, ni, 0.0, T2, ni);
    }
    else
    {
        for (long t = tid; t < long(nb) * ni; t += kScThreads)
            T2[t] = -T1[t];
        __syncthreads();
    }
    // W: [R | -R C] in local mode order
    for (long t = tid; t < long(nb) * nb; t += kScThreads)
    {
        const int r = int(t / nb), c = int(t % nb);
        W[long(r) * nc + a.bm[c]] = a.R ? a.R[t] : (r == c ? 1.0 : 0.0);
    }
    for (long t = tid; t < long(nb) * ni; t += kScThreads)
    {
        const int r = int(t / ni), c = int(t % ni);
        W[long(r) * nc + a.im[c]] = T2[t];
    }
    __syncthreads();
    // -X R^T (ni x nb) into T1 (C is no longer needed)
    if (a.R)
        CtaGemm<false, true>(tiles, ni, nb, nb, -1.0, Z, m, a.R, nb, 0.0, T1, nb);
    else
    {
        for (long t = tid; t < long(ni) * nb; t += kScThreads)
        {
            const int r = int(t / nb), c = int(t % nb);
            T1[t] = -Z[long(r) * m + c];
        }
        __syncthreads();
    }
    // V: rows in local mode order
    for (long t = tid; t < long(nb) * m; t += kScThreads)
    {
        const int r = int(t / m), c = int(t % m);
        V[long(a.bm[r]) * m + c] = c < nb ? (a.R ? a.R[long(c) * nb + r] : (r == c ? 1.0 : 0.0)) : 0.0;
    }
    for (long t = tid; t < long(ni) * m; t += kScThreads)
    {
        const int r = int(t / m), c = int(t % m);
        V[long(a.im[r]) * m + c] = c < nb ? T1[long(r) * nb + c] : Z[long(r) * m + c];
    }
}
} // namespace
} // namespace nkb

using namespace nkb;

extern "C" int nkb_condense(int nelmt, int nc, const double *K, int nb, const int *bm, int ni,
                            const int *im, const double *R, double *S, double *W, double *V,
                            int device, void *stream)
{
    ClearError();
    if (nelmt < 0 || nc < 1 || nb < 1 || ni < 0 || nb + ni != nc || !K || !bm || (ni > 0 && !im) ||
        !S || !W || !V)
        return SetError(NKB_ERR_INVALID, "nkb_condense: bad arguments");
    std::vector<int> seen(nc, 0);
    for (int i = 0; i < nb; ++i)
        if (bm[i] < 0 || bm[i] >= nc || seen[bm[i]]++)
            return SetError(NKB_ERR_INVALID, "nkb_condense: bm is not part of a partition of the modes");
    for (int i = 0; i < ni; ++i)
        if (im[i] < 0 || im[i] >= nc || seen[im[i]]++)
            return SetError(NKB_ERR_INVALID, "nkb_condense: im is not part of a partition of the modes");
    if (nelmt == 0)
        return NKB_OK;
    NKB_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nmax   = std::max(nb, ni);
    // Kii, Z, Kbi (also R S0, nb x nb: room is max(nb * ni, nb * nb)), T1, T2
    const long kbi   = long(nb) * std::max(ni, nb);
    const long wstr  = long(ni) * ni + long(ni) * (nb + ni) + kbi + long(nb) * nmax +
                      long(nmax) * nmax;
    // chunks of at most 2 GB of workspace
    const long chunk = std::max(1L, std::min<long>(nelmt, (2L << 30) / (wstr * 8)));
    int *dbm = nullptr, *dim = nullptr, *derr = nullptr;
    double *dR = nullptr, *ws = nullptr;
    auto release = [&]() {
        cudaFree(dbm);
        cudaFree(dim);
        cudaFree(derr);
        cudaFree(dR);
        cudaFree(ws);
    };
    if (cudaMalloc(&dbm, nb * sizeof(int)) != cudaSuccess ||
        (ni > 0 && cudaMalloc(&dim, ni * sizeof(int)) != cudaSuccess) ||
        cudaMalloc(&derr, sizeof(int)) != cudaSuccess ||
        (R && cudaMalloc(&dR, size_t(nb) * nb * sizeof(double)) != cudaSuccess) ||
        cudaMalloc(&ws, size_t(chunk) * wstr * sizeof(double)) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_condense: workspace of %ld elements", chunk);
    }
    cudaError_t ce = cudaMemcpyAsync(dbm, bm, nb * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess && ni > 0)
        ce = cudaMemcpyAsync(dim, im, ni * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess && R)
        ce = cudaMemcpyAsync(dR, R, size_t(nb) * nb * sizeof(double), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemsetAsync(derr, 0, sizeof(int), s);
    for (long e0 = 0; e0 < nelmt && ce == cudaSuccess; e0 += chunk)
    {
        ScArgs a;
        a.nc = nc;
        a.nb = nb;
        a.ni = ni;
        a.K  = K + e0 * long(nc) * nc;
        a.bm = dbm;
        a.im = dim;
        a.R  = dR;
        a.S  = S + e0 * long(nb) * nb;
        a.W  = W + e0 * long(nb) * nc;
        a.V  = V + e0 * long(nc) * (nb + ni);
        a.ws = ws;
        a.wstride = wstr;
        a.nelmt   = int(std::min(chunk, long(nelmt) - e0));
        a.err     = derr;
        k_condense<<<unsigned(a.nelmt), kScThreads, 0, s>>>(a);
        ce = cudaGetLastError();
    }
    int bad = 0;
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(&bad, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(s);
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_condense: %s", cudaGetErrorString(ce));
    if (bad)
        return SetError(NKB_ERR_INVALID, "nkb_condense: an interior block is not positive definite");
    return NKB_OK;
}

// Assembled blocks of the condensed matrices over mesh entities (the edge and
// face blocks of PreconditionerBlock::BlockPreconditionerCG and the LowEnergy
// block step, PreconditionerLowEnergy.cpp:568-760), built where the
// condensed element matrices are: A_b[i][j] += s_i s_j S_e[l_i][l_j] over the
// contributions (element e, local boundary rows l, signs s) of block b, then
// every block inverted in place.
namespace nkb
{
namespace
{
constexpr int kBlkThreads   = 128;
constexpr int kBlockRowsMax = 256; // the largest block nkb_sys_set_blocks accepts

// one CTA per block (grid-stride); thread t owns the entries t, t + 128, ...
// of its block for every contribution, which it adds in the given order
__global__ void __launch_bounds__(kBlkThreads)
    k_blocks_accumulate(int nblk, const int *__restrict__ bptr, const long *__restrict__ boff,
                        const int *__restrict__ cptr, const int *__restrict__ celm,
                        const long *__restrict__ coff, const int *__restrict__ cloc,
                        const signed char *__restrict__ csgn, const double *__restrict__ S,
                        int nbm, double *__restrict__ A)
{
    for (int b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int n = bptr[b + 1] - bptr[b];
        double *Ab  = A + boff[b];
        for (int c = cptr[b]; c < cptr[b + 1]; ++c)
        {
            const double *Se        = S + long(celm[c]) * nbm * nbm;
            const int *l            = cloc + coff[c];
            const signed char *sg   = csgn + coff[c];
            for (int t = threadIdx.x; t < n * n; t += kBlkThreads)
            {
                const int i = t / n, j = t % n;
                Ab[t] += double(sg[i] * sg[j]) * Se[long(l[i]) * nbm + l[j]];
            }
        }
    }
}

// in-place Gauss-Jordan inversion of each (symmetric positive definite)
// block, without pivoting, then a transpose: the block ends column-major
// (M[j * n + i] = inverse[i][j]); a pivot that is not positive sets *err
__global__ void __launch_bounds__(kBlkThreads)
    k_blocks_invert(int nblk, const int *__restrict__ bptr, const long *__restrict__ boff,
                    double *__restrict__ A, int *err)
{
    __shared__ double col[kBlockRowsMax], row[kBlockRowsMax];
    __shared__ double pinv;
    for (int b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int n = bptr[b + 1] - bptr[b];
        double *M   = A + boff[b];
        for (int k = 0; k < n; ++k)
        {
            if (threadIdx.x == 0)
            {
                const double p = M[long(k) * n + k];
                if (!(p > 0.0))
                    atomicExch(err, 1);
                pinv = p > 0.0 ? 1.0 / p : 0.0;
            }
            __syncthreads();
            const double pi = pinv;
            for (int t = threadIdx.x; t < n; t += kBlkThreads)
            {
                col[t] = M[long(t) * n + k];
                row[t] = t == k ? pi : M[long(k) * n + t] * pi;
            }
            __syncthreads();
            for (int t = threadIdx.x; t < n * n; t += kBlkThreads)
            {
                const int i = t / n, j = t % n;
                if (i == k)
                    M[t] = row[j];
                else
                    M[t] = (j == k ? 0.0 : M[t]) - col[i] * row[j];
            }
            __syncthreads();
        }
        for (int t = threadIdx.x; t < n * n; t += kBlkThreads)
        {
            const int i = t / n, j = t % n;
            if (i < j)
            {
                const double u = M[t];
                M[t]           = M[long(j) * n + i];
                M[long(j) * n + i] = u;
            }
        }
        __syncthreads();
    }
}

int BlockOffsets(const char *fn, int nblk, const int *bptr, std::vector<long> &boff)
{
    if (nblk < 1 || !bptr || bptr[0] != 0)
        return SetError(NKB_ERR_INVALID, "%s: bad block pointers", fn);
    boff.assign(nblk + 1, 0);
    for (int b = 0; b < nblk; ++b)
    {
        const int n = bptr[b + 1] - bptr[b];
        if (n < 1 || n > kBlockRowsMax)
            return SetError(NKB_ERR_INVALID, "%s: block %d has %d rows (1..%d)", fn, b, n,
                            kBlockRowsMax);
        boff[b + 1] = boff[b] + long(n) * n;
    }
    return NKB_OK;
}

int BlockGridSize(int nblk)
{
    return std::max(1, std::min(nblk, 148 * 16));
}
} // namespace
} // namespace nkb

extern "C" int nkb_blocks_accumulate(int nblk, const int *bptr, int ncontrib, const int *cptr,
                                     const int *celm, const int *cloc, const signed char *csgn,
                                     int nelmt, int nbm, const double *S, double *A, int device,
                                     void *stream)
{
    ClearError();
    std::vector<long> boff;
    if (BlockOffsets("nkb_blocks_accumulate", nblk, bptr, boff) != NKB_OK)
        return NKB_ERR_INVALID;
    if (ncontrib < 0 || !cptr || (ncontrib && (!celm || !cloc || !csgn)) || nelmt < 1 || nbm < 1 ||
        !S || !A || cptr[0] != 0 || cptr[nblk] != ncontrib)
        return SetError(NKB_ERR_INVALID, "nkb_blocks_accumulate: bad arguments");
    std::vector<long> coff(size_t(ncontrib) + 1, 0);
    for (int b = 0; b < nblk; ++b)
    {
        if (cptr[b + 1] < cptr[b])
            return SetError(NKB_ERR_INVALID, "nkb_blocks_accumulate: cptr decreases at %d", b);
        const int n = bptr[b + 1] - bptr[b];
        for (int c = cptr[b]; c < cptr[b + 1]; ++c)
        {
            if (celm[c] < 0 || celm[c] >= nelmt)
                return SetError(NKB_ERR_INVALID, "nkb_blocks_accumulate: element %d of "
                                                 "contribution %d outside [0,%d)",
                                celm[c], c, nelmt);
            coff[c + 1] = coff[c] + n;
        }
    }
    const long nloc = coff[ncontrib];
    for (long t = 0; t < nloc; ++t)
        if (cloc[t] < 0 || cloc[t] >= nbm || (csgn[t] != 1 && csgn[t] != -1))
            return SetError(NKB_ERR_INVALID, "nkb_blocks_accumulate: local row %d or sign %d "
                                             "at %ld (rows in [0,%d), signs +-1)",
                            cloc[t], int(csgn[t]), t, nbm);
    if (ncontrib == 0)
        return NKB_OK;
    NKB_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *dbp = nullptr, *dcp = nullptr, *dce = nullptr, *dcl = nullptr;
    long *dbo = nullptr, *dco = nullptr;
    signed char *dcs = nullptr;
    auto release = [&]() {
        cudaFree(dbp);
        cudaFree(dcp);
        cudaFree(dce);
        cudaFree(dcl);
        cudaFree(dbo);
        cudaFree(dco);
        cudaFree(dcs);
    };
    if (cudaMalloc(&dbp, (nblk + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dbo, (nblk + 1) * sizeof(long)) != cudaSuccess ||
        cudaMalloc(&dcp, (nblk + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dce, ncontrib * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dco, (ncontrib + 1) * sizeof(long)) != cudaSuccess ||
        cudaMalloc(&dcl, nloc * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dcs, nloc) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_blocks_accumulate: index arrays");
    }
    cudaError_t ce = cudaMemcpyAsync(dbp, bptr, (nblk + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dbo, boff.data(), (nblk + 1) * sizeof(long), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dcp, cptr, (nblk + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dce, celm, ncontrib * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dco, coff.data(), (ncontrib + 1) * sizeof(long), cudaMemcpyHostToDevice,
                             s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dcl, cloc, nloc * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dcs, csgn, nloc, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
    {
        k_blocks_accumulate<<<BlockGridSize(nblk), kBlkThreads, 0, s>>>(nblk, dbp, dbo, dcp, dce, dco,
                                                                         dcl, dcs, S, nbm, A);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(s);
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_blocks_accumulate: %s", cudaGetErrorString(ce));
    return NKB_OK;
}

extern "C" int nkb_blocks_invert(int nblk, const int *bptr, double *A, int device, void *stream)
{
    ClearError();
    std::vector<long> boff;
    if (BlockOffsets("nkb_blocks_invert", nblk, bptr, boff) != NKB_OK)
        return NKB_ERR_INVALID;
    if (!A)
        return SetError(NKB_ERR_INVALID, "nkb_blocks_invert: bad arguments");
    NKB_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *dbp = nullptr, *derr = nullptr;
    long *dbo = nullptr;
    auto release = [&]() {
        cudaFree(dbp);
        cudaFree(dbo);
        cudaFree(derr);
    };
    if (cudaMalloc(&dbp, (nblk + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dbo, (nblk + 1) * sizeof(long)) != cudaSuccess ||
        cudaMalloc(&derr, sizeof(int)) != cudaSuccess)
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_blocks_invert: index arrays");
    }
    int bad = 0;
    cudaError_t ce = cudaMemcpyAsync(dbp, bptr, (nblk + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dbo, boff.data(), (nblk + 1) * sizeof(long), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemsetAsync(derr, 0, sizeof(int), s);
    if (ce == cudaSuccess)
    {
        k_blocks_invert<<<BlockGridSize(nblk), kBlkThreads, 0, s>>>(nblk, dbp, dbo, A, derr);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(&bad, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(s);
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_blocks_invert: %s", cudaGetErrorString(ce));
    if (bad)
        return SetError(NKB_ERR_INVALID, "nkb_blocks_invert: a block is not positive definite");
    return NKB_OK;
}
