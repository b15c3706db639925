// Prism / Tet Helmholtz, "column" kernels: one element per CTA, one thread
// per (i, j) column of quadrature points holding the whole k direction in
// registers, as the tuned Hex kernel does. The collapsed (Modified_B/C)
// directions change only the mode ranges of the sum-factorisation stages
// (r < nm - p, pairs (p, q)); each stage is one pass over shared memory with
// a k-register array per thread, and the 1-D tables sit in shared memory.
// Arithmetic and the collapsed-vertex / singular-edge corrections are those
// of the generic stages (nkb_generic.cuh), which follow
// BwdTransKernels.hpp:231-403 and IProductKernels.hpp:355-655.
#pragma once

#include "nkb_generic_kernel.cuh"
#include "nkb_tma.cuh"

#include <cstdint>

namespace nkb
{

template <int SHAPE, int NM> struct ColDims
{
    using D                   = SDims<SHAPE, NM>;
    static constexpr int Q0   = D::nq0, Q1 = D::nq1, Q2 = D::nq2;
    static constexpr int NC   = D::nc, NT = D::nt, NP = D::npair;
    static constexpr int T1   = SHAPE == NKB_PRISM ? NM : NP;                    // B1 modes
    static constexpr int T2   = SHAPE == NKB_PRISM ? NP : NC;                    // B2 modes
    static constexpr int TABS = NM * Q0 + T1 * Q1 + T2 * Q2 + Q0 * Q0 + Q1 * Q1 + Q2 * Q2;
    static constexpr int THREADS = (Q0 * Q1 + 31) / 32 * 32;
    // stage scratch: Prism WA [Q2][NM][NM], WB [Q2][Q1][NM]; Tet WA [Q2][NP], WB [Q2][Q1][NM]
    static constexpr int WA   = SHAPE == NKB_PRISM ? Q2 * NM * NM : Q2 * NP;
    static constexpr int WB   = Q2 * Q1 * NM;
    static constexpr int SCR  = (WA > NT ? WA : NT) + (WB > NT ? WB : NT);
    // shared memory (values of T): tables, x, U, scratch (two buffers that
    // also hold V0 and V1)
    static constexpr int SMEM = TABS + ((NC + 1) & ~1) + NT + SCR;
};

template <typename T> __device__ __forceinline__ T ColLd(const T *p)
{
    return __ldg(p);
}

// MODE 0: Helmholtz; 1: Helmholtz with the input gathered from a global
// vector; 2: LinearADR (lambda (W u + W A V'.grad u) as the mass term, packed
// rows 7..9)
template <int SHAPE, int NM, typename T, int MODE>
__global__ void __launch_bounds__(ColDims<SHAPE, NM>::THREADS) k_col_helm(GenArgs<T> a)
{
    constexpr bool GATHER = MODE == 1, ADV = MODE == 2;
    constexpr int NG      = ADV ? 10 : 7; // packed values per point
    using C          = ColDims<SHAPE, NM>;
    constexpr int Q0 = C::Q0, Q1 = C::Q1, Q2 = C::Q2, NC = C::NC, NT = C::NT, NP = C::NP;
    extern __shared__ __align__(16) unsigned char col_raw[];
    T *sm  = reinterpret_cast<T *>(col_raw);
    T *B0  = sm;                      // [p][i]
    T *B1  = B0 + NM * Q0;            // [mode][j]
    T *B2  = B1 + C::T1 * Q1;         // [mode][k]
    T *D0  = B2 + C::T2 * Q2;         // column-major D0[m*Q0 + i] = l_m'(z_i)
    T *D1  = D0 + Q0 * Q0;
    T *D2  = D1 + Q1 * Q1;
    T *x   = D2 + Q2 * Q2;            // coefficients
    T *U   = x + ((NC + 1) & ~1);     // [k][j][i]
    T *S0  = U + NT;                  // scratch 0 (WA, then V0)
    T *S1  = S0 + (C::WA > NT ? C::WA : NT); // scratch 1 (WB, then V1)

    const long e = blockIdx.x;
    if (e >= a.nelmt || (a.skip && *a.skip))
        return;
    const int tid = threadIdx.x;
    const T *G    = a.geo + e * a.gstride;
    if (tid == 0)
        BulkPrefetchL2(G, uint32_t(NG * NT * sizeof(T) + 15) & ~15u);

    for (int l = tid; l < NM * Q0; l += blockDim.x)
        B0[l] = ColLd(a.t.B0 + l);
    for (int l = tid; l < C::T1 * Q1; l += blockDim.x)
        B1[l] = ColLd(a.t.B1 + l);
    for (int l = tid; l < C::T2 * Q2; l += blockDim.x)
        B2[l] = ColLd(a.t.B2 + l);
    for (int l = tid; l < Q0 * Q0; l += blockDim.x)
        D0[l] = ColLd(a.t.D0 + l);
    for (int l = tid; l < Q1 * Q1; l += blockDim.x)
        D1[l] = ColLd(a.t.D1 + l);
    for (int l = tid; l < Q2 * Q2; l += blockDim.x)
        D2[l] = ColLd(a.t.D2 + l);
    // the element's coefficients: every map entry of the thread, then every
    // value, then the stores, so a thread's loads are in flight together
    {
        constexpr int TH  = C::THREADS;
        constexpr int PER = (NC + TH - 1) / TH;
        const T *in0      = GATHER ? a.in : a.in + e * NC;
        int src[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int m = tid + u * TH;
            src[u]      = m < NC ? (GATHER ? a.gmap[e * NC + m] : m) : -1;
        }
        T val[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u)
            val[u] = src[u] >= 0 ? in0[src[u]] : T(0);
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int m = tid + u * TH;
            if (m < NC)
                x[m] = (GATHER && a.gsign) ? val[u] * T(a.gsign[e * NC + m]) : val[u];
        }
    }
    __syncthreads();

    // ---------------- BwdTrans -------------------------------------------
    if constexpr (SHAPE == NKB_PRISM)
    {
        // A: WA[k][p][q] = sum_{r < nm-p} x[(p,q,r)] B2[(p,r)][k], thread (p, q)
        if (tid < NM * NM)
        {
            const int p = tid / NM, q = tid - p * NM;
            const int row = p * NM - (p * (p - 1)) / 2;
            const T *xc   = x + NM * row + q * (NM - p);
            T w[Q2];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
                w[k] = 0;
#pragma unroll
            for (int r = 0; r < NM; ++r)
            {
                if (r < NM - p)
                {
                    const T xv = xc[r];
#pragma unroll
                    for (int k = 0; k < Q2; ++k)
                        w[k] = fma(xv, B2[(row + r) * Q2 + k], w[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < Q2; ++k)
                S0[(k * NM + p) * NM + q] = w[k];
        }
        __syncthreads();
        // B: WB[k][j][p] = sum_q WA[k][p][q] B1[q][j], thread (p, j)
        if (tid < NM * Q1)
        {
            const int p = tid / Q1, j = tid - p * Q1;
            T b1[NM];
#pragma unroll
            for (int q = 0; q < NM; ++q)
                b1[q] = B1[q * Q1 + j];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T s = 0;
#pragma unroll
                for (int q = 0; q < NM; ++q)
                    s = fma(S0[(k * NM + p) * NM + q], b1[q], s);
                S1[(k * Q1 + j) * NM + p] = s;
            }
        }
    }
    else
    {
        // A: WA[k][pair(p,q)] = sum_{r < nm-p-q} x[(p,q,r)] B2[(p,q,r)][k], thread pair
        if (tid < NP)
        {
            int p = 0, rem = tid;
#pragma unroll
            for (int pp = 0; pp < NM; ++pp)
            {
                if (rem >= NM - p)
                {
                    rem -= NM - p;
                    ++p;
                }
            }
            const int q = rem;
            int m0      = 0;
#pragma unroll
            for (int pp = 0; pp < NM; ++pp)
                if (pp < p)
                    m0 += (NM - pp) * (NM - pp + 1) / 2;
            m0 += q * (NM - p) - (q * (q - 1)) / 2;
            T w[Q2];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
                w[k] = 0;
#pragma unroll
            for (int r = 0; r < NM; ++r)
            {
                if (r < NM - p - q)
                {
                    const T xv = x[m0 + r];
#pragma unroll
                    for (int k = 0; k < Q2; ++k)
                        w[k] = fma(xv, B2[(m0 + r) * Q2 + k], w[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < Q2; ++k)
                S0[k * NP + tid] = w[k];
        }
        __syncthreads();
        // B: WB[k][j][p] = sum_{q < nm-p} WA[k][pair(p,q)] B1[pair(p,q)][j], thread (p, j)
        if (tid < NM * Q1)
        {
            const int p = tid / Q1, j = tid - p * Q1;
            const int pr = p * NM - (p * (p - 1)) / 2;
            T b1[NM];
#pragma unroll
            for (int q = 0; q < NM; ++q)
                b1[q] = q < NM - p ? B1[(pr + q) * Q1 + j] : T(0);
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T s = 0;
#pragma unroll
                for (int q = 0; q < NM; ++q)
                    if (q < NM - p)
                        s = fma(S0[k * NP + pr + q], b1[q], s);
                S1[(k * Q1 + j) * NM + p] = s;
            }
        }
    }
    __syncthreads();

    const int i    = tid % Q0, j = tid / Q0;
    const bool act = j < Q1;
    T u[Q2];
    if (act)
    {
        // C: u[k] = sum_p WB[k][j][p] B0[p][i] + collapsed corrections
        T b0[NM];
#pragma unroll
        for (int p = 0; p < NM; ++p)
            b0[p] = B0[p * Q0 + i];
        T cadd[Q2];
        if constexpr (SHAPE == NKB_PRISM)
        {
            // singular edge: phi_1q1 through phi_0q1 (BwdTransKernels.hpp:388-399)
            T cj = 0;
#pragma unroll
            for (int q = 0; q < NM; ++q)
                cj = fma(B1[q * Q1 + j], x[q * NM + 1], cj);
            const T f = cj * b0[1];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
                cadd[k] = B2[Q2 + k] * f;
        }
        else
        {
            // top vertex, bottom vertex, singular edge (BwdTransKernels.hpp:293-324)
            const T a0 = b0[0], a1 = b0[1], bb0 = B1[j], bb1 = B1[Q1 + j];
            const T top = fma(a1, bb1, fma(a1, bb0, a0 * bb1)) * x[1];
            const T ab  = a1 * bb1;
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T ev = x[NM] * B2[k];
#pragma unroll
                for (int r = 1; r < NM - 1; ++r)
                    ev = fma(x[NM + r], B2[(r + 1) * Q2 + k], ev);
                cadd[k] = fma(ab, ev, top * B2[Q2 + k]);
            }
        }
#pragma unroll
        for (int k = 0; k < Q2; ++k)
        {
            const T *wb = S1 + (k * Q1 + j) * NM;
            T s         = 0;
#pragma unroll
            for (int p = 0; p < NM; ++p)
                s = fma(wb[p], b0[p], s);
            u[k]                    = s + cadd[k];
            U[(k * Q1 + j) * Q0 + i] = u[k];
        }
    }
    __syncthreads();

    // ---------------- gradient, metric, transposed gradient ----------------
    T f[Q2], v2[Q2];
    if (act)
    {
        T d0[Q0], d1[Q1];
#pragma unroll
        for (int m = 0; m < Q0; ++m)
            d0[m] = D0[m * Q0 + i];
#pragma unroll
        for (int m = 0; m < Q1; ++m)
            d1[m] = D1[m * Q1 + j];
        const T lam = a.lambda;
#pragma unroll
        for (int k = 0; k < Q2; ++k)
        {
            const int q  = (k * Q1 + j) * Q0 + i;
            const T *row = U + (k * Q1 + j) * Q0;
            T g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
            for (int m = 0; m < Q0; ++m)
                g0 = fma(d0[m], row[m], g0);
#pragma unroll
            for (int m = 0; m < Q1; ++m)
                g1 = fma(d1[m], U[(k * Q1 + m) * Q0 + i], g1);
#pragma unroll
            for (int m = 0; m < Q2; ++m)
                g2 = fma(D2[m * Q2 + k], u[m], g2);
            const T W = ColLd(G + q), G00 = ColLd(G + NT + q), G11 = ColLd(G + 2 * NT + q);
            const T G22 = ColLd(G + 3 * NT + q), G01 = ColLd(G + 4 * NT + q);
            const T G02 = ColLd(G + 5 * NT + q), G12 = ColLd(G + 6 * NT + q);
            S0[q] = fma(G02, g2, fma(G01, g1, G00 * g0));
            S1[q] = fma(G12, g2, fma(G11, g1, G01 * g0));
            v2[k] = fma(G22, g2, fma(G12, g1, G02 * g0));
            if (ADV)
            {
                const T adv = fma(ColLd(G + 9 * NT + q), g2,
                                  fma(ColLd(G + 8 * NT + q), g1, ColLd(G + 7 * NT + q) * g0));
                f[k] = lam * fma(W, u[k], adv);
            }
            else
            {
                f[k] = lam * W * u[k];
            }
        }
    }
    __syncthreads();
    if (act)
    {
        T t0[Q0], t1[Q1];
#pragma unroll
        for (int m = 0; m < Q0; ++m)
            t0[m] = D0[i * Q0 + m];
#pragma unroll
        for (int m = 0; m < Q1; ++m)
            t1[m] = D1[j * Q1 + m];
#pragma unroll
        for (int k = 0; k < Q2; ++k)
        {
            const T *row = S0 + (k * Q1 + j) * Q0;
            T s          = f[k];
#pragma unroll
            for (int m = 0; m < Q0; ++m)
                s = fma(t0[m], row[m], s);
#pragma unroll
            for (int m = 0; m < Q1; ++m)
                s = fma(t1[m], S1[(k * Q1 + m) * Q0 + i], s);
#pragma unroll
            for (int m = 0; m < Q2; ++m)
                s = fma(D2[k * Q2 + m], v2[m], s);
            f[k] = s;
        }
    }
    __syncthreads();
    if (act)
    {
#pragma unroll
        for (int k = 0; k < Q2; ++k)
            U[(k * Q1 + j) * Q0 + i] = f[k];
    }
    __syncthreads();

    // ---------------- raw inner product ----------------------------------
    // IA: WA2[k][j][p] = sum_i F[k][j][i] B0[p][i], thread (p, j)
    if (tid < NM * Q1)
    {
        const int p = tid / Q1, jj = tid - p * Q1;
        T b0r[Q0];
#pragma unroll
        for (int ii = 0; ii < Q0; ++ii)
            b0r[ii] = B0[p * Q0 + ii];
#pragma unroll
        for (int k = 0; k < Q2; ++k)
        {
            const T *row = U + (k * Q1 + jj) * Q0;
            T s          = 0;
#pragma unroll
            for (int ii = 0; ii < Q0; ++ii)
                s = fma(row[ii], b0r[ii], s);
            S0[(k * Q1 + jj) * NM + p] = s;
        }
    }
    __syncthreads();
    T *y = a.out0 + e * NC;
    if constexpr (SHAPE == NKB_PRISM)
    {
        // IB: wb[k] = sum_j WA2[k][j][p] B1[q][j], thread (p, q); kept in
        // registers and also stored for the singular-edge fold
        T wb[Q2];
        const int p = tid / NM, q = tid - (tid / NM) * NM;
        if (tid < NM * NM)
        {
            T b1r[Q1];
#pragma unroll
            for (int jj = 0; jj < Q1; ++jj)
                b1r[jj] = B1[q * Q1 + jj];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T s = 0;
#pragma unroll
                for (int jj = 0; jj < Q1; ++jj)
                    s = fma(S0[(k * Q1 + jj) * NM + p], b1r[jj], s);
                wb[k]                      = s;
                S1[(k * NM + q) * NM + p] = s;
            }
        }
        __syncthreads();
        // IC: y[(p,q,r)] = sum_k wb[k] B2[(p,r)][k] (+ fold of phi_1q1 into phi_0q1)
        if (tid < NM * NM)
        {
            const int row = p * NM - (p * (p - 1)) / 2;
            T *yc         = y + NM * row + q * (NM - p);
#pragma unroll
            for (int r = 0; r < NM; ++r)
            {
                if (r < NM - p)
                {
                    T s = 0;
#pragma unroll
                    for (int k = 0; k < Q2; ++k)
                        s = fma(wb[k], B2[(row + r) * Q2 + k], s);
                    if (p == 0 && r == 1)
                    {
#pragma unroll
                        for (int k = 0; k < Q2; ++k)
                            s = fma(S1[(k * NM + q) * NM + 1], B2[Q2 + k], s);
                    }
                    yc[r] = s;
                }
            }
        }
    }
    else
    {
        // IB: wb[k] = sum_j WA2[k][j][p] B1[pair(p,q)][j], thread pair; the
        // correction columns c0[k], c1[k] by threads NP and NP + 1
        constexpr int CB = 2 * Q2; // c0 then c1 in S1
        int p = 0, rem = tid;
#pragma unroll
        for (int pp = 0; pp < NM; ++pp)
        {
            if (rem >= NM - p)
            {
                rem -= NM - p;
                ++p;
            }
        }
        const int q = rem;
        T wb[Q2];
        if (tid < NP)
        {
            T b1r[Q1];
#pragma unroll
            for (int jj = 0; jj < Q1; ++jj)
                b1r[jj] = B1[tid * Q1 + jj];
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T s = 0;
#pragma unroll
                for (int jj = 0; jj < Q1; ++jj)
                    s = fma(S0[(k * Q1 + jj) * NM + p], b1r[jj], s);
                wb[k] = s;
            }
        }
        else if (tid < NP + 2)
        {
            // c0[k] = sum_j B1[1][j] a0 + B1[0][j] a1; c1[k] = sum_j B1[1][j] a1
            const int which = tid - NP;
#pragma unroll
            for (int k = 0; k < Q2; ++k)
            {
                T s = 0;
#pragma unroll
                for (int jj = 0; jj < Q1; ++jj)
                {
                    const T a0 = S0[(k * Q1 + jj) * NM + 0], a1 = S0[(k * Q1 + jj) * NM + 1];
                    if (which == 0)
                        s = fma(B1[Q1 + jj], a0, fma(B1[jj], a1, s));
                    else
                        s = fma(B1[Q1 + jj], a1, s);
                }
                S1[which * Q2 + k] = s;
            }
        }
        (void)CB;
        __syncthreads();
        if (tid < NP)
        {
            int m0 = 0;
#pragma unroll
            for (int pp = 0; pp < NM; ++pp)
                if (pp < p)
                    m0 += (NM - pp) * (NM - pp + 1) / 2;
            m0 += q * (NM - p) - (q * (q - 1)) / 2;
            const T *c0 = S1, *c1 = S1 + Q2;
#pragma unroll
            for (int r = 0; r < NM; ++r)
            {
                if (r < NM - p - q)
                {
                    const int m = m0 + r;
                    T s         = 0;
#pragma unroll
                    for (int k = 0; k < Q2; ++k)
                        s = fma(wb[k], B2[m * Q2 + k], s);
                    // top vertex, bottom vertex, singular edge (IProductKernels.hpp:456-513)
                    if (m == 1)
                    {
#pragma unroll
                        for (int k = 0; k < Q2; ++k)
                            s = fma(B2[Q2 + k], c0[k] + c1[k], s);
                    }
                    else if (m == NM)
                    {
#pragma unroll
                        for (int k = 0; k < Q2; ++k)
                            s = fma(B2[k], c1[k], s);
                    }
                    else if (m > NM && m < 2 * NM - 1)
                    {
                        const int rr = m - NM;
#pragma unroll
                        for (int k = 0; k < Q2; ++k)
                            s = fma(B2[(rr + 1) * Q2 + k], c1[k], s);
                    }
                    y[m] = s;
                }
            }
        }
    }
}

// one element per CTA; kNotCovered unless a standard Prism/Tet point set
template <int SHAPE, int NM, typename T>
int LaunchColShapeNM(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s, bool gather)
{
    using C           = ColDims<SHAPE, NM>;
    const size_t smem = size_t(C::SMEM) * sizeof(T);
    if (smem > 200 * 1024)
        return kNotCovered;
    const int mode = op->optype == NKB_LINEAR_ADR ? 2 : (gather ? 1 : 0);
    if (mode == 2 && gather)
        return kNotCovered;
    auto kern = mode == 2 ? k_col_helm<SHAPE, NM, T, 2>
                          : (mode == 1 ? k_col_helm<SHAPE, NM, T, 1> : k_col_helm<SHAPE, NM, T, 0>);
    static size_t s_set[3] = {48 * 1024, 48 * 1024, 48 * 1024};
    size_t &set            = s_set[mode];
    if (smem > set)
    {
        NKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        set = smem;
    }
    if (op->nelmt > 0)
        kern<<<unsigned(op->nelmt), C::THREADS, smem, s>>>(a);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

template <int SHAPE, typename T>
int LaunchColShape(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s, bool gather)
{
    switch (op->nm)
    {
#define NKB_CS(N)                                                                                  \
    case N: return LaunchColShapeNM<SHAPE, N, T>(op, a, s, gather);
        NKB_CS(2) NKB_CS(3) NKB_CS(4) NKB_CS(5) NKB_CS(6) NKB_CS(7) NKB_CS(8) NKB_CS(9)
        NKB_CS(10) NKB_CS(11)
#undef NKB_CS
        default: return kNotCovered;
    }
}

template <typename T> int LaunchColHelm(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s)
{
    const int nm = op->nm;
    if (op->nq[0] != nm + 1)
        return kNotCovered;
    const bool gather = a.gmap != nullptr;
    if (op->shape == NKB_PRISM && op->nq[1] == nm + 1 && op->nq[2] == nm)
        return LaunchColShape<NKB_PRISM, T>(op, a, s, gather);
    if (op->shape == NKB_TET && op->nq[1] == nm && op->nq[2] == nm)
        return LaunchColShape<NKB_TET, T>(op, a, s, gather);
    return kNotCovered;
}

} // namespace nkb
