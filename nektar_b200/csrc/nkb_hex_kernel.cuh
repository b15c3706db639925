// The tuned Hex Helmholtz kernel template (see nkb_hex.cu for the design) and
// its variant launcher. Included by nkb_hex_f64.cu / nkb_hex_f32.cu, which
// instantiate it per precision, and declared for nkb_hex.cu.
#pragma once

#include "nkb_op.h"
#include "nkb_tma.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace nkb
{

int SmCount(int device); // multiprocessors of a device (nkb_hex.cu)
// CTAs of a kernel that stay resident on one SM at `threads` threads and
// `smem` bytes of dynamic shared memory, from its register and shared-memory
// use (nkb_hex.cu)
int ResidentCtas(const void *fn, int threads, size_t smem);


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
    int *err;           // [0] error word, [1] first bound of bounded waits (0: kMaxPolls)
    const int *skip;    // optional: nonzero -> nothing to do (converged CG)
};

// kernel modes (the last template argument of the Hex kernels)
enum
{
    kModeLocal  = 0,
    kModeGather = 1,
    kModeAdv    = 2
};

// geometry staging
enum
{
    kGeoTma    = 0, // the element's whole geometry by one bulk TMA copy into shared memory
    kGeoStream = 1, // coalesced loads into registers, one k-plane ahead
    kGeoTma2   = 2, // persistent CTAs: the next element group's geometry copied into a
                    // second buffer while the current group computes
    kGeoTmaS   = 3  // as kGeoTma, with element groups of at most 48 KB and 128 registers
                    // per thread (more CTAs per SM)
};

__host__ __device__ constexpr int RoundUp(int a, int b)
{
    return (a + b - 1) / b * b;
}

template <int NQ, int EPB> __host__ __device__ constexpr int HexThreads()
{
    return RoundUp(EPB * NQ * NQ, 32);
}

template <typename T, int NM, int NQ> constexpr int HexTabBytes()
{
    return RoundUp(16 + (3 * NM * NQ + NQ * (NQ + 1)) * int(sizeof(T)), 128);
}

// shared memory of one CTA (the TMA variant adds EPB element geometry blocks)
// element stride of the work regions: nq^3 rounded up to an even count, so every
// element's region (and every even-length row in it) starts 16-byte aligned
template <int NQ> __host__ __device__ constexpr int HexRegion()
{
    return NQ * NQ * NQ + ((NQ * NQ * NQ) & 1);
}

template <typename T, int NM, int NQ, int GEO, int EPB> size_t HexSmem(long gstride)
{
    const size_t nbuf = (GEO == kGeoTma || GEO == kGeoTmaS) ? 1 : (GEO == kGeoTma2 ? 2 : 0);
    return size_t(HexTabBytes<T, NM, NQ>()) +
           size_t(EPB) * (nbuf * size_t(gstride) + 3 * HexRegion<NQ>()) * sizeof(T);
}

// 1-D tables passed by value as a kernel parameter: entries read with
// compile-time indices (the uniform, register-direction contractions) become
// constant-bank operands of the FMAs instead of shared-memory loads.
template <typename T, int NM, int NQ> struct HexConst
{
    T B0[NM * NQ], B1[NM * NQ], B2[NM * NQ]; // B[p*NQ + i] = phi_p(z_i)
    T D[NQ * NQ];                            // D[i*NQ + m] = l_m'(z_i)
};

template <typename T> struct Vec2;
template <> struct Vec2<double>
{
    using type = double2;
};
template <> struct Vec2<float>
{
    using type = float2;
};

// sum_m c[m] v[m] over a shared-memory row, 16-byte (FP64) loads when the row
// length is even (rows are then aligned)
template <typename T, int N>
__device__ __forceinline__ T DotRow(const T *__restrict__ row, const T (&c)[N], T s)
{
    if constexpr (N % 2 == 0)
    {
        using V = typename Vec2<T>::type;
#pragma unroll
        for (int m = 0; m < N; m += 2)
        {
            const V v = *reinterpret_cast<const V *>(row + m);
            s         = fma(c[m], v.x, s);
            s         = fma(c[m + 1], v.y, s);
        }
    }
    else
    {
#pragma unroll
        for (int m = 0; m < N; ++m)
            s = fma(c[m], row[m], s);
    }
    return s;
}

template <typename T, int NQ, int GEO, int EPB> __host__ __device__ constexpr int HexMinBlocks()
{
    // resident CTAs per SM the register allocation must allow: a register
    // budget per thread of 160 (nq <= 8), 168 (nq <= 10) or 255; the streamed
    // variants up to nq = 10 (no shared-memory geometry buffer, so registers
    // set the occupancy) take 128
    constexpr int regs = (GEO == kGeoStream && NQ <= 10) || GEO == kGeoTmaS
                             ? 128
                             : (NQ <= 8 ? 160 : (NQ <= 10 ? 168 : 255));
    constexpr int b    = 65536 / (HexThreads<NQ, EPB>() * regs);
    return b < 1 ? 1 : b;
}

// MODE: kModeLocal (Helmholtz), kModeGather (Helmholtz, input gathered from
// a global vector), kModeAdv (LinearADR: lambda (W u + W A V'.grad u) as the
// mass term, packed rows 7..9)
template <typename T, int NM, int NQ, int GEO, int EPB, int MODE>
__global__ void __launch_bounds__(HexThreads<NQ, EPB>(), (HexMinBlocks<T, NQ, GEO, EPB>()))
    k_hex_helm(HexArgs<T> a, const __grid_constant__ HexConst<T, NM, NQ> c)
{
    constexpr bool GATHER = MODE == kModeGather, ADV = MODE == kModeAdv;
    constexpr int NG      = ADV ? 10 : 7; // packed values per point
    constexpr int NQ2 = NQ * NQ, NQ3 = NQ2 * NQ, NC = NM * NM * NM, NQP = NQ + 1;
    constexpr int NMP = NM + (NM & 1); // coefficient rows padded to an even length
    constexpr int RS  = HexRegion<NQ>(); // element stride of the work regions (even)
    static_assert(RS % 2 == 0 && NMP % 2 == 0, "vector loads need even strides");
    static_assert(HexTabBytes<T, NM, NQ>() % 16 == 0, "work regions must start 16-byte aligned");
    static_assert(NM * NM * NMP <= RS && NM * NQ * NQ <= RS, "regions too small");
    constexpr bool TMA = GEO == kGeoTma || GEO == kGeoTma2 || GEO == kGeoTmaS;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem); // one per geometry buffer
    T *sB0         = reinterpret_cast<T *>(smem + 16);
    T *sB1        = sB0 + NM * NQ;
    T *sB2        = sB1 + NM * NQ;
    T *sD         = sB2 + NM * NQ; // sD[i*NQP + m] = D(i, m) = l_m'(z_i)
    const long GS = a.gstride;
    T *geob       = reinterpret_cast<T *>(smem + HexTabBytes<T, NM, NQ>());
    T *us         = geob + (GEO == kGeoTma2 ? 2 : (TMA ? 1 : 0)) * EPB * GS; // GS % 4 == 0
    T *v0s        = us + EPB * RS;
    T *v1s        = v0s + EPB * RS;

    const int tid       = threadIdx.x;
    const long ngroups  = (long(a.nelmt) + EPB - 1) / EPB;
    // the persistent variant walks groups blockIdx.x, + gridDim.x, ...; the
    // others take one group each
    const long gstep = GEO == kGeoTma2 ? long(gridDim.x) : ngroups;
    if (long(blockIdx.x) >= ngroups || (a.skip && *a.skip))
        return;
    auto group_bytes = [&](long grp) {
        const long ng = min(long(EPB), long(a.nelmt) - grp * EPB);
        return uint32_t(ng * GS * long(sizeof(T)));
    };
    if (TMA && tid == 0)
    {
        MbarInit(&bars[0], 1);
        if (GEO == kGeoTma2)
            MbarInit(&bars[1], 1);
        const uint32_t bytes = group_bytes(blockIdx.x);
        MbarArriveExpectTx(&bars[0], bytes);
        BulkG2S(geob, a.geo + long(blockIdx.x) * EPB * GS, bytes, &bars[0]);
    }

    const int le   = tid / NQ2;
    const int ij   = tid - le * NQ2;
    const int i    = ij % NQ, j = ij / NQ;
    const int lec  = le < EPB ? le : 0;
    const int eoff = lec * RS;
    T *xs = v0s + eoff, *As = v1s + eoff, *u_ = us + eoff, *v0 = v0s + eoff, *v1 = v1s + eoff;

    for (int t = tid; t < NM * NQ; t += blockDim.x)
    {
        sB0[t] = c.B0[t];
        sB1[t] = c.B1[t];
        sB2[t] = c.B2[t];
    }
    for (int t = tid; t < NQ2; t += blockDim.x)
    {
        const int r = t / NQ, cc = t - r * NQ;
        sD[r * NQP + cc] = c.D[r * NQ + cc];
    }
    int it = 0; // groups done by this CTA
    for (long grp = blockIdx.x; grp < ngroups; grp += gstep, ++it)
    {
    const long e0  = grp * EPB;
    const int ne   = int(min(long(EPB), long(a.nelmt) - e0));
    bool act       = le < ne;
    const int cur  = GEO == kGeoTma2 ? (it & 1) : 0;
    T *geo         = geob + cur * EPB * GS;
    if (GEO == kGeoTma2 && tid == 0 && grp + gstep < ngroups)
    {
        // the other buffer was last read by the previous group, which every
        // thread has finished (the barrier ending that group)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t bytes = group_bytes(grp + gstep);
        MbarArriveExpectTx(&bars[cur ^ 1], bytes);
        BulkG2S(geob + (cur ^ 1) * EPB * GS, a.geo + (grp + gstep) * EPB * GS, bytes,
                &bars[cur ^ 1]);
    }
    if (GEO == kGeoStream && tid == 0)
    {
        // the CTA's whole geometry requested from DRAM at once (into L2); the
        // per-plane loads below then hit L2
        BulkPrefetchL2(a.geo + e0 * GS, uint32_t(ne * GS * long(sizeof(T))));
    }
    // streamed geometry: plane 0 requested before any arithmetic
    const T *Gg = a.geo + (e0 + lec) * GS;
    T gc[NG];
    if (GEO == kGeoStream && act)
    {
        const int q0 = j * NQ + i;
#pragma unroll
        for (int cc = 0; cc < NG; ++cc)
            gc[cc] = __ldg(Gg + cc * NQ3 + q0);
    }
    // coefficients into the v0 region, rows (r, q) padded to NMP (NM^2 NMP <= NQ3):
    // every map entry of the thread first, then every value, then the stores,
    // so the loads of one thread are in flight together
    {
        constexpr int TH  = HexThreads<NQ, EPB>();
        constexpr int PER = (EPB * NC + TH - 1) / TH;
        const int nall    = ne * NC;
        // gathered: the global index; local: the offset in the group
        const T *in0 = GATHER ? a.in : a.in + e0 * NC;
        int src[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int t = tid + u * TH;
            src[u]      = t < nall ? (GATHER ? a.gmap[e0 * NC + t] : t) : -1;
        }
        T val[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u)
            val[u] = src[u] >= 0 ? in0[src[u]] : T(0);
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int t = tid + u * TH;
            if (t < nall)
            {
                T v = val[u];
                if (GATHER && a.gsign)
                    v *= T(a.gsign[e0 * NC + t]);
                const int lt = t / NC;
                const int m  = t - lt * NC;
                const int rq = m / NM;
                v0s[lt * RS + rq * NMP + (m - rq * NM)] = v;
            }
        }
    }
    __syncthreads();

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
            const T *xr = xs + (r * NM + j) * NMP;
            T s         = 0;
            using V     = typename Vec2<T>::type;
#pragma unroll
            for (int p = 0; p < NMP; p += 2)
            {
                const V v = *reinterpret_cast<const V *>(xr + p);
                s         = fma(v.x, b0[p], s);
                if (p + 1 < NM)
                    s = fma(v.y, b0[p + 1], s);
            }
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
                s = fma(c.B2[r * NQ + k], bv[r], s);
            ur[k]                     = s;
            u_[(k * NQ + j) * NQ + i] = s;
        }
    }
    __syncthreads();

    // TMA geometry must have landed: bounded wait by every thread (use
    // it >> 1 of buffer cur)
    if (TMA && !MbarWaitBounded(&bars[cur], uint32_t((it >> 1) & 1), a.err, 1, WaitPolls(a.err)))
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
        const T *G = geo + lec * GS;
#pragma unroll
        for (int k = 0; k < NQ; ++k)
        {
            const int q = (k * NQ + j) * NQ + i;
            T gn[NG];
            if (GEO == kGeoStream && k + 1 < NQ)
            {
#pragma unroll
                for (int cc = 0; cc < NG; ++cc)
                    gn[cc] = __ldg(Gg + cc * NQ3 + q + NQ2);
            }
            T g1 = 0, g2 = 0;
            const T g0   = DotRow<T, NQ>(u_ + (k * NQ + j) * NQ, d0, T(0));
            const T *col = u_ + k * NQ2 + i;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                g1 = fma(d1[m], col[m * NQ], g1);
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                g2 = fma(c.D[k * NQ + m], ur[m], g2);
            T W, G00, G11, G22, G01, G02, G12, A0 = 0, A1 = 0, A2 = 0;
            if (TMA)
            {
                W   = G[q];
                G00 = G[NQ3 + q];
                G11 = G[2 * NQ3 + q];
                G22 = G[3 * NQ3 + q];
                G01 = G[4 * NQ3 + q];
                G02 = G[5 * NQ3 + q];
                G12 = G[6 * NQ3 + q];
                if (ADV)
                {
                    A0 = G[7 * NQ3 + q];
                    A1 = G[8 * NQ3 + q];
                    A2 = G[9 * NQ3 + q];
                }
            }
            else
            {
                W   = gc[0];
                G00 = gc[1];
                G11 = gc[2];
                G22 = gc[3];
                G01 = gc[4];
                G02 = gc[5];
                G12 = gc[6];
                if (ADV)
                {
                    A0 = gc[7 % NG];
                    A1 = gc[8 % NG];
                    A2 = gc[9 % NG];
                }
            }
            v0[q]  = fma(G02, g2, fma(G01, g1, G00 * g0));
            v1[q]  = fma(G12, g2, fma(G11, g1, G01 * g0));
            v2r[k] = fma(G22, g2, fma(G12, g1, G02 * g0));
            if (ADV)
                fr[k] = a.lambda * fma(W, ur[k], fma(A2, g2, fma(A1, g1, A0 * g0)));
            else
                fr[k] = a.lambda * W * ur[k];
            if (GEO == kGeoStream && k + 1 < NQ)
            {
#pragma unroll
                for (int cc = 0; cc < NG; ++cc)
                    gc[cc] = gn[cc];
            }
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
            T s          = DotRow<T, NQ>(v0 + (k * NQ + j) * NQ, dt0, fr[k]);
            const T *col = v1 + k * NQ2 + i;
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                s = fma(dt1[m], col[m * NQ], s);
#pragma unroll
            for (int m = 0; m < NQ; ++m)
                s = fma(c.D[m * NQ + k], v2r[m], s);
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
                s = fma(c.B2[r * NQ + k], fr[k], s);
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
            o[(r * NM + j) * NM + i] = DotRow<T, NQ>(v0 + (r * NM + j) * NQ, b0c, T(0));
        }
    }
    __syncthreads(); // the work regions and this group's geometry buffer are free again
    }
}

// ---------------------------------------------------------------------------
// variants, autotuning and dispatch
// ---------------------------------------------------------------------------

enum
{
    kVariantGeneric = 0,
    kVariantHexHelm = 1
};

// candidate (geometry staging, elements per CTA) of the tuned Hex kernel
} // namespace nkb

#include "nkb_hex_tc.cuh"

namespace nkb
{

// 0: TMA-staged geometry; 1, 2: streamed geometry, 1 or 2 elements per CTA;
// 3: FP64 tensor cores (DMMA, nq <= 8, FP64 arithmetic for both storage
//    precisions; nkb_hex_mma.cuh); 4: the same with two warps per element
//    (nkb_hex_mma2.cuh); 5: fifth-generation tensor cores (tcgen05, TF32
//    high/low operands, FP32 accumulation; FP32 operators, nm 2..9;
//    nkb_hex_tc.cuh); 6: persistent CTAs with the geometry double-buffered
//    (the next element group's bulk copy in flight while the current one
//    computes); 7: TMA-staged geometry in element groups of at most 48 KB,
//    128 registers per thread (more, smaller CTAs per SM than variant 0);
//    8: the same in groups of at most 72 KB (offered where that holds more
//    elements than variant 7's groups: at nq = 6, four elements of 36
//    threads fill 144 of 160 lanes where two fill 72 of 96)
constexpr int kNumHexVariants = 9;

// elements per CTA of the double-buffered variant: two geometry buffers and
// three work regions per element in at most 72 KB (three CTAs per SM)
template <typename T, int NQ> constexpr int Tma2Epb()
{
    constexpr int per = (2 * (7 * NQ * NQ * NQ + 4) + 3 * (NQ * NQ * NQ + 1)) * int(sizeof(T));
    constexpr int e   = (72 * 1024) / per;
    constexpr int lim = 512 / (NQ * NQ);
    constexpr int v   = e < lim ? e : lim;
    return v < 1 ? 1 : (v > 8 ? 8 : v);
}

template <typename T, int NQ> constexpr int TmaEpb()
{
    constexpr int per = (10 * NQ * NQ * NQ + 4) * int(sizeof(T));
    constexpr int e   = (90 * 1024) / per;
    constexpr int lim = 512 / (NQ * NQ);
    constexpr int v   = e < lim ? e : lim;
    return v < 1 ? 1 : (v > 8 ? 8 : v);
}

// elements per CTA of variant 7: groups of at most 48 KB (one element when a
// single element needs more)
template <typename T, int NQ, int KB = 48> constexpr int TmaSmallEpb()
{
    constexpr int per = (10 * NQ * NQ * NQ + 4) * int(sizeof(T));
    constexpr int e   = (KB * 1024) / per;
    constexpr int lim = 512 / (NQ * NQ);
    constexpr int v   = e < lim ? e : lim;
    return v < 1 ? 1 : (v > 8 ? 8 : v);
}

template <typename T, int NM, int NQ> static HexConst<T, NM, NQ> MakeHexConst(const nkb_op *op)
{
    HexConst<T, NM, NQ> c;
    for (int t = 0; t < NM * NQ; ++t)
    {
        c.B0[t] = T(op->hB[0][t]);
        c.B1[t] = T(op->hB[1][t]);
        c.B2[t] = T(op->hB[2][t]);
    }
    // host D is column-major (D[m*NQ + i] = l_m'(z_i)); the table is row-major
    for (int i = 0; i < NQ; ++i)
        for (int m = 0; m < NQ; ++m)
            c.D[i * NQ + m] = T(op->hD[0][size_t(m) * NQ + i]);
    return c;
}

// the kernel mode of a launch: gathered Helmholtz, LinearADR (local only; -1
// if gathered) or local Helmholtz
inline int HexMode(const nkb_op *op, bool gather)
{
    if (op->optype == NKB_LINEAR_ADR)
        return gather ? -1 : kModeAdv;
    return gather ? kModeGather : kModeLocal;
}

template <typename T, int NM, int GEO, int EPB>
static int HexVariantLaunch(const nkb_op *op, const HexArgs<T> &a, bool gather, cudaStream_t s,
                            bool set_attr)
{
    constexpr int NQ   = NM + 1;
    const size_t bytes = HexSmem<T, NM, NQ, GEO, EPB>(op->gstride);
    if (bytes > 227 * 1024 || HexThreads<NQ, EPB>() > 1024)
        return SetError(NKB_ERR_UNSUPPORTED, "Hex variant needs %zu bytes of shared memory", bytes);
    const int mode = HexMode(op, gather);
    if (mode < 0)
        return SetError(NKB_ERR_UNSUPPORTED, "LinearADR has no gathered Hex kernel");
    if (set_attr)
    {
        // the limit of each mode's kernel covers every operator that may
        // launch it: Helmholtz packs 7 geometry values per point, LinearADR
        // 10 (another operator's set-up must not lower it under this one's)
        const long nt = long(NQ) * NQ * NQ;
        const size_t hb = HexSmem<T, NM, NQ, GEO, EPB>((7 * nt + 3) & ~3L);
        const size_t ab = HexSmem<T, NM, NQ, GEO, EPB>((10 * nt + 3) & ~3L);
        NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm<T, NM, NQ, GEO, EPB, kModeLocal>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(std::max(hb, bytes))));
        NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm<T, NM, NQ, GEO, EPB, kModeGather>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(std::max(hb, bytes))));
        if (ab <= 227 * 1024)
            NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm<T, NM, NQ, GEO, EPB, kModeAdv>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(std::max(ab, bytes))));
        return NKB_OK;
    }
    long nb = (long(op->nelmt) + EPB - 1) / EPB;
    if (nb == 0)
        return NKB_OK;
    const HexConst<T, NM, NQ> c = MakeHexConst<T, NM, NQ>(op);
    const unsigned th           = HexThreads<NQ, EPB>();
    if (GEO == kGeoTma2)
    {
        // persistent grid: every CTA that stays resident walks its groups
        const void *fn = mode == kModeGather
                             ? (const void *)k_hex_helm<T, NM, NQ, GEO, EPB, kModeGather>
                             : (mode == kModeAdv ? (const void *)k_hex_helm<T, NM, NQ, GEO, EPB, kModeAdv>
                                                 : (const void *)k_hex_helm<T, NM, NQ, GEO, EPB, kModeLocal>);
        const long resident = long(ResidentCtas(fn, int(th), bytes)) * SmCount(op->device);
        nb                  = nb < resident ? nb : resident;
    }
    if (mode == kModeGather)
        k_hex_helm<T, NM, NQ, GEO, EPB, kModeGather><<<unsigned(nb), th, bytes, s>>>(a, c);
    else if (mode == kModeAdv)
        k_hex_helm<T, NM, NQ, GEO, EPB, kModeAdv><<<unsigned(nb), th, bytes, s>>>(a, c);
    else
        k_hex_helm<T, NM, NQ, GEO, EPB, kModeLocal><<<unsigned(nb), th, bytes, s>>>(a, c);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

template <typename TV, int NM>
static int HexMmaLaunch(const nkb_op *op, const HexArgs<TV> &a, bool gather, cudaStream_t s,
                        bool set_attr);
template <typename TV, int NM>
static int HexMma2Launch(const nkb_op *op, const HexArgs<TV> &a, bool gather, cudaStream_t s,
                         bool set_attr);

template <int NM>
static int HexTcLaunch(const nkb_op *op, const HexArgs<float> &a, bool gather, cudaStream_t s,
                       bool set_attr)
{
    constexpr int NQ = NM + 1;
    using Dm         = TcDims<NM, NQ>;
    if (!op->tc_tab || op->optype != NKB_HELMHOLTZ)
        return SetError(NKB_ERR_UNSUPPORTED, "tensor-core Hex kernel: FP32 Helmholtz only");
    const size_t bytes = TcSmemBytes<NM, NQ>(op->tc_bytes);
    if (bytes > 227 * 1024)
        return SetError(NKB_ERR_UNSUPPORTED, "tensor-core Hex kernel needs %zu bytes of shared memory",
                        bytes);
    if (set_attr)
    {
        NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm_tc<NM, NQ, kModeLocal>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
        NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm_tc<NM, NQ, kModeGather>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
        return NKB_OK;
    }
    const long ntile = (long(op->nelmt) + Dm::EPT - 1) / Dm::EPT;
    if (ntile == 0)
        return NKB_OK;
    // persistent grid: the CTAs per SM the launch bounds were built for
    // (shared and tensor memory allow that many; ncu confirms the register
    // limit), each walking its tiles
    const long resident = long(Dm::MIN_CTAS) * SmCount(op->device);
    const long nb       = ntile < resident ? ntile : resident;
    TcTables tt;
    tt.tab   = op->tc_tab;
    tt.bytes = op->tc_bytes;
    for (int d = 0; d < 3; ++d)
    {
        tt.tb[d]  = op->tc_tb[d];
        tt.tbt[d] = op->tc_tbt[d];
    }
    if (gather)
        k_hex_helm_tc<NM, NQ, kModeGather><<<unsigned(nb), 128, bytes, s>>>(a, tt);
    else
        k_hex_helm_tc<NM, NQ, kModeLocal><<<unsigned(nb), 128, bytes, s>>>(a, tt);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

template <typename T, int NM>
static int HexLaunch(const nkb_op *op, const HexArgs<T> &a, bool gather, cudaStream_t s, int variant,
                     bool set_attr)
{
    constexpr int NQ = NM + 1;
    if (variant == 5)
    {
        if constexpr (std::is_same<T, float>::value && NM >= kTcMinNm && NM <= kTcMaxNm)
            return HexTcLaunch<NM>(op, a, gather, s, set_attr);
        else
            return SetError(NKB_ERR_UNSUPPORTED, "tensor-core Hex kernel: FP32 operators, nm 2..9");
    }
    if (variant == 3)
        return HexMmaLaunch<T, NM>(op, a, gather, s, set_attr);
    if (variant == 4)
        return HexMma2Launch<T, NM>(op, a, gather, s, set_attr);
    switch (variant)
    {
        case 0:
            return HexVariantLaunch<T, NM, kGeoTma, TmaEpb<T, NQ>()>(op, a, gather, s, set_attr);
        case 6:
            if constexpr (NQ <= 9)
                return HexVariantLaunch<T, NM, kGeoTma2, Tma2Epb<T, NQ>()>(op, a, gather, s, set_attr);
            else
                return SetError(NKB_ERR_UNSUPPORTED, "double-buffered Hex variant: nq <= 9");
        case 1:
            return HexVariantLaunch<T, NM, kGeoStream, 1>(op, a, gather, s, set_attr);
        case 7:
            return HexVariantLaunch<T, NM, kGeoTmaS, TmaSmallEpb<T, NQ>()>(op, a, gather, s,
                                                                           set_attr);
        case 8:
            if constexpr (TmaSmallEpb<T, NQ, 72>() > TmaSmallEpb<T, NQ>())
                return HexVariantLaunch<T, NM, kGeoTmaS, TmaSmallEpb<T, NQ, 72>()>(op, a, gather,
                                                                                   s, set_attr);
            else
                return SetError(NKB_ERR_UNSUPPORTED,
                                "Hex variant 8: no larger group than variant 7 at nq=%d", NQ);
        default:
            return HexVariantLaunch<T, NM, kGeoStream, 2>(op, a, gather, s, set_attr);
    }
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

template <typename T>
int HexLaunchT(const nkb_op *op, const HexArgs<T> &a, bool gather, cudaStream_t s, int variant,
               bool set_attr)
{
#define NKB_CALL(N) HexLaunch<T, N>(op, a, gather, s, variant, set_attr)
    NKB_HEX_SWITCH(op->nm, NKB_CALL)
#undef NKB_CALL
}


} // namespace nkb

#include "nkb_hex_mma.cuh"
