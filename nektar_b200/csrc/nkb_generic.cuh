// Shape-generic sum-factorisation stages for one element held in shared
// memory. Every stage computes one output entry per call from a flat local
// index; the kernels in nkb_ops.cu spread the entries of all elements of a
// CTA over its threads and separate the stages with __syncthreads().
//
// Layouts (per element):
//   x   coefficients (Hex: p fastest, then q, r; Prism/Tet: r fastest inside
//       (p, q) with the Modified_B/C truncation, BwdTransKernels.hpp:171-186,
//       245-266, 348-363)
//   u   values at the nq0 x nq1 x nq2 points, i fastest
//   B0, B1, B2  1-D tables, mode-major with the point index fastest
//       (Basis::GetBdata); Prism B2 is Modified_B, Tet B1 Modified_B and B2
//       Modified_C (Basis.cpp:499-644)
//   D0, D1, D2  column-major collocation derivatives, D[k*nq + i] = l_k'(z_i)
//
// BwdTrans follows BwdTransKernels.hpp:160-403 (Hex / Tet / Prism, with the
// collapsed-vertex "correct" terms of the Modified_A direction). The inner
// product is the reference's IProductKernels.hpp:271-655 applied to a field
// that already carries the quadrature weights and Jacobian (raw inner
// product), including the Tet vertex / singular-edge and Prism singular-edge
// corrections.
#pragma once

#include "nkb_internal.h"

namespace nkb
{

struct Dims
{
    int nm, nq0, nq1, nq2;
    int nc, nt;
    int npair; // Tet: nm(nm+1)/2 (p,q) pairs
    int wsz;   // size of each of the two sum-factorisation scratch arrays
};

// Compile-time sizes of the meshes' standard point sets (nq0 = nm + 1 GLL;
// Prism nq2 = nm, Tet nq1 = nq2 = nm Gauss-Radau): the stage functions above
// take either these or the runtime Dims; with these every loop bound, index
// division and scratch offset is a constant.
template <int SHAPE, int NM> struct SDims
{
    static constexpr int nm    = NM;
    static constexpr int nq0   = NM + 1;
    static constexpr int nq1   = SHAPE == NKB_TET ? NM : NM + 1;
    static constexpr int nq2   = SHAPE == NKB_HEX ? NM + 1 : NM;
    static constexpr int nc    = SHAPE == NKB_HEX     ? NM * NM * NM
                                 : SHAPE == NKB_PRISM ? NM * NM * (NM + 1) / 2
                                                      : NM * (NM + 1) * (NM + 2) / 6;
    static constexpr int nt    = nq0 * nq1 * nq2;
    static constexpr int npair = NM * (NM + 1) / 2;
    static constexpr int wsz   = nq0 * nq0 * nq0 + 2 * nq2 + nq0 * nq0;
};

template <typename T> struct Tabs
{
    const T *B0, *B1, *B2;
    const T *D0, *D1, *D2;
};

// (p, q) pair index of the Tet Modified_B table: sum_{p'<p} (nm - p') + q
__device__ __forceinline__ int TetPair(int nm, int p, int q)
{
    return p * nm - (p * (p - 1)) / 2 + q;
}
// first coefficient of the Tet (p, q, 0) column
__device__ __forceinline__ int TetCoeff(int nm, int p, int q)
{
    // sum_{p'<p} T(nm-p') + sum_{q'<q} (nm - p - q'), T(n) = n(n+1)/2
    int off = 0;
    for (int pp = 0; pp < p; ++pp)
        off += (nm - pp) * (nm - pp + 1) / 2;
    return off + q * (nm - p) - (q * (q - 1)) / 2;
}
// Prism (p, r) row of the Modified_B table: sum_{p'<p} (nm - p')
__device__ __forceinline__ int PrismRow(int nm, int p)
{
    return p * nm - (p * (p - 1)) / 2;
}

// ---------------------------------------------------------------------------
// BwdTrans: x (nc) -> u (nt), scratch wa, wb
// ---------------------------------------------------------------------------
template <int SHAPE> struct Bwd;

template <> struct Bwd<NKB_HEX>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nm * d.nm * d.nq0; }
    template <class D> __device__ static int SizeB(const D &d) { return d.nm * d.nq1 * d.nq0; }
    template <class D, typename T>
    __device__ static void A(const D &d, const Tabs<T> &t, const T *x, T *wa, int l)
    {
        // wa[(r*nm + q)*nq0 + i] = sum_p x[(r*nm+q)*nm + p] B0[p][i]
        int i = l % d.nq0, rq = l / d.nq0;
        const T *xr = x + rq * d.nm;
        T s = 0;
        for (int p = 0; p < d.nm; ++p)
            s = fma(xr[p], t.B0[p * d.nq0 + i], s);
        wa[l] = s;
    }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *, const T *wa, T *wb, int l)
    {
        // wb[(r*nq1 + j)*nq0 + i] = sum_q wa[(r*nm+q)*nq0+i] B1[q][j]
        int i = l % d.nq0, j = (l / d.nq0) % d.nq1, r = l / (d.nq0 * d.nq1);
        T s = 0;
        for (int q = 0; q < d.nm; ++q)
            s = fma(wa[(r * d.nm + q) * d.nq0 + i], t.B1[q * d.nq1 + j], s);
        wb[l] = s;
    }
    template <class D, typename T>
    __device__ static void C(const D &d, const Tabs<T> &t, const T *, const T *wb, T *u, int l)
    {
        int ij = l % (d.nq0 * d.nq1), k = l / (d.nq0 * d.nq1);
        T s = 0;
        for (int r = 0; r < d.nm; ++r)
            s = fma(wb[r * d.nq0 * d.nq1 + ij], t.B2[r * d.nq2 + k], s);
        u[l] = s;
    }
};

template <> struct Bwd<NKB_PRISM>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nq2 * d.nm * d.nm; }
    template <class D> __device__ static int SizeB(const D &d) { return d.nq2 * d.nq1 * d.nm; }
    template <class D, typename T>
    __device__ static void A(const D &d, const Tabs<T> &t, const T *x, T *wa, int l)
    {
        // wa[(k*nm + p)*nm + q] = sum_{r<nm-p} x[(p,q,r)] B2[(p,r)][k]
        int q = l % d.nm, p = (l / d.nm) % d.nm, k = l / (d.nm * d.nm);
        int row = PrismRow(d.nm, p);
        const T *xc = x + d.nm * row + q * (d.nm - p);
        T s = 0;
        for (int r = 0; r < d.nm - p; ++r)
            s = fma(xc[r], t.B2[(row + r) * d.nq2 + k], s);
        wa[l] = s;
    }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *, const T *wa, T *wb, int l)
    {
        // wb[(k*nq1 + j)*nm + p] = sum_q wa[(k*nm+p)*nm+q] B1[q][j]
        int p = l % d.nm, j = (l / d.nm) % d.nq1, k = l / (d.nm * d.nq1);
        const T *a = wa + (k * d.nm + p) * d.nm;
        T s = 0;
        for (int q = 0; q < d.nm; ++q)
            s = fma(a[q], t.B1[q * d.nq1 + j], s);
        wb[l] = s;
    }
    template <class D, typename T>
    __device__ static void C(const D &d, const Tabs<T> &t, const T *x, const T *wb, T *u, int l)
    {
        int i = l % d.nq0, j = (l / d.nq0) % d.nq1, k = l / (d.nq0 * d.nq1);
        const T *b = wb + (k * d.nq1 + j) * d.nm;
        T s = 0;
        for (int p = 0; p < d.nm; ++p)
            s = fma(b[p], t.B0[p * d.nq0 + i], s);
        // singular edge: phi_1q1 contributes through phi_0q1 (BwdTransKernels.hpp:388-399)
        T c = 0;
        for (int q = 0; q < d.nm; ++q)
            c = fma(t.B1[q * d.nq1 + j], x[q * d.nm + 1], c);
        s = fma(t.B2[d.nq2 + k] * t.B0[d.nq0 + i], c, s);
        u[l] = s;
    }
};

template <> struct Bwd<NKB_TET>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nq2 * d.npair; }
    template <class D> __device__ static int SizeB(const D &d) { return d.nq2 * d.nq1 * d.nm; }
    template <class D, typename T>
    __device__ static void A(const D &d, const Tabs<T> &t, const T *x, T *wa, int l)
    {
        // wa[k*npair + pair(p,q)] = sum_{r<nm-p-q} x[(p,q,r)] B2[(p,q,r)][k]
        int pq = l % d.npair, k = l / d.npair;
        int p = 0, rem = pq;
        while (rem >= d.nm - p)
        {
            rem -= d.nm - p;
            ++p;
        }
        int q = rem;
        int m0 = TetCoeff(d.nm, p, q);
        T s = 0;
        for (int r = 0; r < d.nm - p - q; ++r)
            s = fma(x[m0 + r], t.B2[(m0 + r) * d.nq2 + k], s);
        wa[l] = s;
    }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *, const T *wa, T *wb, int l)
    {
        // wb[(k*nq1 + j)*nm + p] = sum_{q<nm-p} wa[k*npair + pair(p,q)] B1[pair(p,q)][j]
        int p = l % d.nm, j = (l / d.nm) % d.nq1, k = l / (d.nm * d.nq1);
        int pr = TetPair(d.nm, p, 0);
        const T *a = wa + k * d.npair + pr;
        T s = 0;
        for (int q = 0; q < d.nm - p; ++q)
            s = fma(a[q], t.B1[(pr + q) * d.nq1 + j], s);
        wb[l] = s;
    }
    template <class D, typename T>
    __device__ static void C(const D &d, const Tabs<T> &t, const T *x, const T *wb, T *u, int l)
    {
        int i = l % d.nq0, j = (l / d.nq0) % d.nq1, k = l / (d.nq0 * d.nq1);
        const T *b = wb + (k * d.nq1 + j) * d.nm;
        T s = 0;
        for (int p = 0; p < d.nm; ++p)
            s = fma(b[p], t.B0[p * d.nq0 + i], s);
        // collapsed top vertex, bottom vertex and singular edge
        // (BwdTransKernels.hpp:293-324)
        const T a0 = t.B0[i], a1 = t.B0[d.nq0 + i];
        const T b0 = t.B1[j], b1 = t.B1[d.nq1 + j];
        T top = fma(a1, b1, fma(a1, b0, a0 * b1)) * t.B2[d.nq2 + k];
        s = fma(top, x[1], s);
        T e = x[d.nm] * t.B2[k];
        for (int r = 1; r < d.nm - 1; ++r)
            e = fma(x[d.nm + r], t.B2[(r + 1) * d.nq2 + k], e);
        s = fma(a1 * b1, e, s);
        u[l] = s;
    }
};

// ---------------------------------------------------------------------------
// Raw inner product: f (nt, already weighted) -> y (nc), scratch wa, wb
// ---------------------------------------------------------------------------
template <int SHAPE> struct Ipr;

// stage A common to all shapes: wa[(k*nq1 + j)*nm + p] = sum_i f[kji] B0[p][i]
template <class D, typename T>
__device__ __forceinline__ void IprStageA(const D &d, const Tabs<T> &t, const T *f, T *wa, int l)
{
    int p = l % d.nm, kj = l / d.nm;
    const T *fr = f + kj * d.nq0;
    T s = 0;
    for (int i = 0; i < d.nq0; ++i)
        s = fma(fr[i], t.B0[p * d.nq0 + i], s);
    wa[l] = s;
}

template <> struct Ipr<NKB_HEX>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nq2 * d.nq1 * d.nm; }
    template <class D> __device__ static int SizeB(const D &d) { return d.nq2 * d.nm * d.nm; }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *wa, T *wb, int l)
    {
        // wb[(k*nm + q)*nm + p] = sum_j wa[(k*nq1+j)*nm + p] B1[q][j]
        int p = l % d.nm, q = (l / d.nm) % d.nm, k = l / (d.nm * d.nm);
        T s = 0;
        for (int j = 0; j < d.nq1; ++j)
            s = fma(wa[(k * d.nq1 + j) * d.nm + p], t.B1[q * d.nq1 + j], s);
        wb[l] = s;
    }
    template <class D, typename T>
    __device__ static T C(const D &d, const Tabs<T> &t, const T *wb, int m)
    {
        int pq = m % (d.nm * d.nm), r = m / (d.nm * d.nm);
        T s = 0;
        for (int k = 0; k < d.nq2; ++k)
            s = fma(wb[k * d.nm * d.nm + pq], t.B2[r * d.nq2 + k], s);
        return s;
    }
};

template <> struct Ipr<NKB_PRISM>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nq2 * d.nq1 * d.nm; }
    template <class D> __device__ static int SizeB(const D &d) { return d.nq2 * d.nm * d.nm; }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *wa, T *wb, int l)
    {
        Ipr<NKB_HEX>::B(d, t, wa, wb, l);
    }
    template <class D, typename T>
    __device__ static T C(const D &d, const Tabs<T> &t, const T *wb, int m)
    {
        // m -> (p, q, r), r < nm - p
        int p = 0, rem = m;
        while (rem >= d.nm * (d.nm - p))
        {
            rem -= d.nm * (d.nm - p);
            ++p;
        }
        int q = rem / (d.nm - p), r = rem % (d.nm - p);
        int row = PrismRow(d.nm, p) + r;
        T s = 0;
        for (int k = 0; k < d.nq2; ++k)
            s = fma(wb[(k * d.nm + q) * d.nm + p], t.B2[row * d.nq2 + k], s);
        if (p == 0 && r == 1)
        {
            // singular edge (IProductKernels.hpp:606-654): phi_1q1 folded into phi_0q1
            for (int k = 0; k < d.nq2; ++k)
                s = fma(wb[(k * d.nm + q) * d.nm + 1], t.B2[d.nq2 + k], s);
        }
        return s;
    }
};

template <> struct Ipr<NKB_TET>
{
    template <class D> __device__ static int SizeA(const D &d) { return d.nq2 * d.nq1 * d.nm; }
    // wb holds nq2*npair pair sums followed by the two correction columns c0, c1
    template <class D> __device__ static int SizeB(const D &d) { return d.nq2 * (d.npair + 2); }
    template <class D, typename T>
    __device__ static void B(const D &d, const Tabs<T> &t, const T *wa, T *wb, int l)
    {
        const int np = d.nq2 * d.npair;
        if (l < np)
        {
            int pq = l % d.npair, k = l / d.npair;
            int p = 0, rem = pq;
            while (rem >= d.nm - p)
            {
                rem -= d.nm - p;
                ++p;
            }
            T s = 0;
            for (int j = 0; j < d.nq1; ++j)
                s = fma(wa[(k * d.nq1 + j) * d.nm + p], t.B1[pq * d.nq1 + j], s);
            wb[l] = s;
        }
        else
        {
            // c0[k] = sum_j B1[1][j] a0 + B1[0][j] a1 ; c1[k] = sum_j B1[1][j] a1
            int which = (l - np) / d.nq2, k = (l - np) % d.nq2;
            T s = 0;
            for (int j = 0; j < d.nq1; ++j)
            {
                const T a0 = wa[(k * d.nq1 + j) * d.nm + 0];
                const T a1 = wa[(k * d.nq1 + j) * d.nm + 1];
                if (which == 0)
                    s = fma(t.B1[d.nq1 + j], a0, fma(t.B1[j], a1, s));
                else
                    s = fma(t.B1[d.nq1 + j], a1, s);
            }
            wb[l] = s;
        }
    }
    template <class D, typename T>
    __device__ static T C(const D &d, const Tabs<T> &t, const T *wb, int m)
    {
        int p = 0, rem = m;
        while (rem >= (d.nm - p) * (d.nm - p + 1) / 2)
        {
            rem -= (d.nm - p) * (d.nm - p + 1) / 2;
            ++p;
        }
        int q = 0;
        while (rem >= d.nm - p - q)
        {
            rem -= d.nm - p - q;
            ++q;
        }
        const int pq = TetPair(d.nm, p, q);
        T s = 0;
        for (int k = 0; k < d.nq2; ++k)
            s = fma(wb[k * d.npair + pq], t.B2[m * d.nq2 + k], s);
        // top vertex, bottom vertex, singular edge (IProductKernels.hpp:456-513)
        const T *c0 = wb + d.nq2 * d.npair, *c1 = c0 + d.nq2;
        if (m == 1)
        {
            for (int k = 0; k < d.nq2; ++k)
                s = fma(t.B2[d.nq2 + k], c0[k] + c1[k], s);
        }
        else if (m == d.nm)
        {
            for (int k = 0; k < d.nq2; ++k)
                s = fma(t.B2[k], c1[k], s);
        }
        else if (m > d.nm && m < 2 * d.nm - 1)
        {
            const int r = m - d.nm;
            for (int k = 0; k < d.nq2; ++k)
                s = fma(t.B2[(r + 1) * d.nq2 + k], c1[k], s);
        }
        return s;
    }
};

// ---------------------------------------------------------------------------
// collocation derivatives on the nq0 x nq1 x nq2 grid
// ---------------------------------------------------------------------------
template <class D, typename T>
__device__ __forceinline__ void Grad(const D &d, const Tabs<T> &t, const T *u, int l, T &g0,
                                     T &g1, T &g2)
{
    int i = l % d.nq0, j = (l / d.nq0) % d.nq1, k = l / (d.nq0 * d.nq1);
    const T *row = u + (k * d.nq1 + j) * d.nq0;
    T s0 = 0, s1 = 0, s2 = 0;
    for (int m = 0; m < d.nq0; ++m)
        s0 = fma(t.D0[m * d.nq0 + i], row[m], s0);
    const T *col = u + k * d.nq1 * d.nq0 + i;
    for (int m = 0; m < d.nq1; ++m)
        s1 = fma(t.D1[m * d.nq1 + j], col[m * d.nq0], s1);
    const T *pil = u + j * d.nq0 + i;
    for (int m = 0; m < d.nq2; ++m)
        s2 = fma(t.D2[m * d.nq2 + k], pil[m * d.nq0 * d.nq1], s2);
    g0 = s0;
    g1 = s1;
    g2 = s2;
}

// sum_a D_a^T v_a at point l
template <class D, typename T>
__device__ __forceinline__ T GradT(const D &d, const Tabs<T> &t, const T *v0, const T *v1,
                                   const T *v2, int l)
{
    int i = l % d.nq0, j = (l / d.nq0) % d.nq1, k = l / (d.nq0 * d.nq1);
    const T *row = v0 + (k * d.nq1 + j) * d.nq0;
    T s = 0;
    for (int m = 0; m < d.nq0; ++m)
        s = fma(t.D0[i * d.nq0 + m], row[m], s);
    const T *col = v1 + k * d.nq1 * d.nq0 + i;
    for (int m = 0; m < d.nq1; ++m)
        s = fma(t.D1[j * d.nq1 + m], col[m * d.nq0], s);
    const T *pil = v2 + j * d.nq0 + i;
    for (int m = 0; m < d.nq2; ++m)
        s = fma(t.D2[k * d.nq2 + m], pil[m * d.nq0 * d.nq1], s);
    return s;
}

} // namespace nkb
