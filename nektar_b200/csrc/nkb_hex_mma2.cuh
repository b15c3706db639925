// Hex Helmholtz on the FP64 tensor cores, two warps per element (variant 4).
// Same arithmetic, cube layout and pipeline as k_hex_helm_mma (variant 3,
// nkb_hex_mma.cuh); each warp of a pair computes half of the 8 row tiles of
// every contraction and half of the metric points, and the pair meets at a
// named barrier between stages. Half the work per warp needs fewer
// registers, so more warps stay resident to hide shared-memory and DMMA
// latency. When the three directions share one basis (always for the
// standard Hex), one set of table fragments serves all of them (ISO).
#pragma once

// included at the end of nkb_hex_mma.cuh
#include "nkb_hex_mma.cuh"

namespace nkb
{

constexpr int kMma2Pairs = 2; // elements (warp pairs) per CTA

__device__ __forceinline__ void PairSync(int pair)
{
    // the two warps of one element (64 threads) meet; shared-memory writes
    // before the barrier are visible after it
    asm volatile("bar.sync %0, 64;\n" ::"r"(1 + pair) : "memory");
}

// the contraction of Contract<AX, ACC, TIN> restricted to tiles [tile0, tile0 + 4)
template <int AX, bool ACC, typename TIN = double>
__device__ __forceinline__ void Contract4(const TIN *__restrict__ in, double *__restrict__ out,
                                          const double (&bf)[2], int g, int t, int tile0)
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int tile = tile0 + i;
        int ia0, ia1, io0, io1;
        if (AX == 0)
        {
            ia0 = CubeIdx(tile, g, t);
            ia1 = CubeIdx(tile, g, t + 4);
            io0 = CubeIdx(tile, g, 2 * t);
            io1 = io0 + 1;
        }
        else if (AX == 1)
        {
            ia0 = CubeIdx(tile, t, g);
            ia1 = CubeIdx(tile, t + 4, g);
            io0 = CubeIdx(tile, 2 * t, g);
            io1 = CubeIdx(tile, 2 * t + 1, g);
        }
        else
        {
            ia0 = CubeIdx(t, tile, g);
            ia1 = CubeIdx(t + 4, tile, g);
            io0 = CubeIdx(2 * t, tile, g);
            io1 = CubeIdx(2 * t + 1, tile, g);
        }
        double c0 = 0.0, c1 = 0.0;
        if (AX == 0)
        {
            double2 *o2 = reinterpret_cast<double2 *>(out + io0);
            if (ACC)
            {
                const double2 v = *o2;
                c0              = v.x;
                c1              = v.y;
            }
            Dmma(c0, c1, double(in[ia0]), bf[0]);
            Dmma(c0, c1, double(in[ia1]), bf[1]);
            *o2 = make_double2(c0, c1);
        }
        else
        {
            if (ACC)
            {
                c0 = out[io0];
                c1 = out[io1];
            }
            Dmma(c0, c1, double(in[ia0]), bf[0]);
            Dmma(c0, c1, double(in[ia1]), bf[1]);
            out[io0] = c0;
            out[io1] = c1;
        }
    }
}

// the lane's 8 cube positions of this warp's half: pos = lane + 32 s, s in [8h, 8h + 8)
template <int NM, bool GATHER, typename TV>
__device__ __forceinline__ void LoadMap8(const HexArgs<TV> &a, long e, int lane, int h, int (&idx)[8])
{
    constexpr int NC = NM * NM * NM;
#pragma unroll
    for (int s = 0; s < 8; ++s)
    {
        const int pos = lane + 32 * (8 * h + s);
        const int cc = pos >> 6, bb = (pos >> 3) & 7, aa = pos & 7;
        const int m  = (cc * NM + bb) * NM + aa;
        const bool real = aa < NM && bb < NM && cc < NM;
        idx[s]          = real ? (GATHER ? __ldg(a.gmap + e * NC + m) : m) : -1;
    }
}

template <int NM, bool GATHER, typename TV>
__device__ __forceinline__ void FetchCoeffs8(const HexArgs<TV> &a, long e, int lane, int h,
                                             const int (&idx)[8], TV *x)
{
    constexpr int NC = NM * NM * NM;
#pragma unroll
    for (int s = 0; s < 8; ++s)
    {
        if (idx[s] < 0)
            continue;
        const int pos = lane + 32 * (8 * h + s);
        TV *dst       = x + CubeIdx(pos >> 6, (pos >> 3) & 7, pos & 7);
        if (!GATHER)
        {
            CpAsync(dst, a.in + e * NC + idx[s]);
        }
        else if (!a.gsign)
        {
            CpAsync(dst, a.in + idx[s]);
        }
        else
        {
            const int m = ((pos >> 6) * NM + ((pos >> 3) & 7)) * NM + (pos & 7);
            *dst        = TV(double(__ldg(a.in + idx[s])) * __ldg(a.gsign + e * NC + m));
        }
    }
    CpAsyncCommit();
}

template <typename TV, int NM, int NQ, int MODE, bool ISO>
__global__ void __launch_bounds__(64 * kMma2Pairs, 4)
    k_hex_helm_mma2(HexArgs<TV> a, const __grid_constant__ HexConst<double, NM, NQ> c)
{
    constexpr bool GATHER = MODE == kModeGather, ADV = MODE == kModeAdv;
    constexpr int NG      = ADV ? 10 : 7; // packed values per point
    static_assert(NQ <= 8 && NM < NQ, "the DMMA Hex kernel covers nq <= 8");
    constexpr int NQ2 = NQ * NQ, NQ3 = NQ2 * NQ, NC = NM * NM * NM;
    extern __shared__ __align__(16) double msm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = warp >> 1, h = warp & 1, tile0 = 4 * h;
    const int g = lane >> 2, t = lane & 3;
    const long npairs = long(gridDim.x) * kMma2Pairs;
    long e            = long(blockIdx.x) * kMma2Pairs + pair;
    if (e >= a.nelmt || (a.skip && *a.skip))
        return; // both warps of the pair leave together
    double *c0 = msm + pair * kMmaCubes * kMmaCube + kMmaCube, *c1 = c0 + kMmaCube,
           *c2 = c1 + kMmaCube;
    TV *xc = reinterpret_cast<TV *>(c0 - kMmaCube);
    const uint32_t gbytes = uint32_t(NG * NQ3 * sizeof(TV) + 15) & ~15u;

    MmaTabs<NM, NQ> f;
    LoadMmaTabs<NM, NQ>(c, f, g, t);
    const double(&bw0)[2] = f.bw[0];
    const double(&bw1)[2] = ISO ? f.bw[0] : f.bw[1];
    const double(&bw2)[2] = ISO ? f.bw[0] : f.bw[2];
    const double(&ip0)[2] = f.ip[0];
    const double(&ip1)[2] = ISO ? f.ip[0] : f.ip[1];
    const double(&ip2)[2] = ISO ? f.ip[0] : f.ip[2];
    const double lam = double(a.lambda);

    for (int pos = lane + 32 * h; pos < kMmaCube; pos += 64)
        xc[pos] = TV(0);
    // the zero fill interleaves the two warps' positions, the fetch splits them
    // in halves: without this barrier a late zero store of one warp can land
    // on a coefficient the other warp's copy has already written
    PairSync(pair);
    int idx[8];
    LoadMap8<NM, GATHER, TV>(a, e, lane, h, idx);
    FetchCoeffs8<NM, GATHER, TV>(a, e, lane, h, idx, xc);
    if (e + npairs < a.nelmt)
        LoadMap8<NM, GATHER, TV>(a, e + npairs, lane, h, idx);

    for (; e < a.nelmt; e += npairs)
    {
        const TV *__restrict__ G = a.geo + e * a.gstride;
        if (lane == 0 && h == 0)
            BulkPrefetchL2(G, gbytes);
        CpAsyncWaitAll();
        PairSync(pair);
        Contract4<0, false, TV>(xc, c1, bw0, g, t, tile0);
        PairSync(pair);
        const long en = e + npairs;
        if (en < a.nelmt)
        {
            FetchCoeffs8<NM, GATHER, TV>(a, en, lane, h, idx, xc);
            if (en + npairs < a.nelmt)
                LoadMap8<NM, GATHER, TV>(a, en + npairs, lane, h, idx);
        }
        Contract4<1, false>(c1, c0, bw1, g, t, tile0);
        PairSync(pair);
        Contract4<2, false>(c0, c1, bw2, g, t, tile0);
        PairSync(pair);
        Contract4<0, false>(c1, c0, f.dg, g, t, tile0);
        Contract4<1, false>(c1, c2, f.dg, g, t, tile0);
        double z[4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const int tile = tile0 + i;
            z[i][0] = z[i][1] = 0.0;
            Dmma(z[i][0], z[i][1], c1[CubeIdx(t, tile, g)], f.dg[0]);
            Dmma(z[i][0], z[i][1], c1[CubeIdx(t + 4, tile, g)], f.dg[1]);
        }
        PairSync(pair);
#pragma unroll
        for (int i = 0; i < 4; ++i) // batches of the two points (c = 2t, 2t + 1) of one tile
        {
            const int tile = tile0 + i;
            double gv[2][NG];
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
            {
                const int cc    = 2 * t + hh;
                const bool real = cc < NQ && tile < NQ && g < NQ;
                const int q     = real ? (cc * NQ + tile) * NQ + g : 0;
#pragma unroll
                for (int k = 0; k < NG; ++k)
                    gv[hh][k] = real ? double(__ldg(G + k * NQ3 + q)) : 0.0;
            }
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
            {
                const int ci    = CubeIdx(2 * t + hh, tile, g);
                const double x0 = c0[ci], x1 = c2[ci], x2 = z[i][hh];
                const double W = gv[hh][0], G00 = gv[hh][1], G11 = gv[hh][2], G22 = gv[hh][3];
                const double G01 = gv[hh][4], G02 = gv[hh][5], G12 = gv[hh][6];
                c0[ci]          = fma(G02, x2, fma(G01, x1, G00 * x0));
                c2[ci]          = fma(G12, x2, fma(G11, x1, G01 * x0));
                const double v2 = fma(G22, x2, fma(G12, x1, G02 * x0));
                if (ADV)
                {
                    const double adv = fma(gv[hh][9 % NG], x2,
                                           fma(gv[hh][8 % NG], x1, gv[hh][7 % NG] * x0));
                    z[i][hh]         = lam * fma(W, c1[ci], adv);
                }
                else
                {
                    z[i][hh] = lam * W * c1[ci];
                }
                c1[ci]          = v2;
            }
        }
        PairSync(pair);
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const int tile = tile0 + i;
            Dmma(z[i][0], z[i][1], c1[CubeIdx(t, tile, g)], f.dt[0]);
            Dmma(z[i][0], z[i][1], c1[CubeIdx(t + 4, tile, g)], f.dt[1]);
        }
        PairSync(pair);
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const int tile = tile0 + i;
            c1[CubeIdx(2 * t, tile, g)]     = z[i][0];
            c1[CubeIdx(2 * t + 1, tile, g)] = z[i][1];
        }
        PairSync(pair);
        Contract4<0, true>(c0, c1, f.dt, g, t, tile0);
        PairSync(pair);
        Contract4<1, true>(c2, c1, f.dt, g, t, tile0);
        PairSync(pair);
        Contract4<2, false>(c1, c0, ip2, g, t, tile0);
        PairSync(pair);
        Contract4<1, false>(c0, c2, ip1, g, t, tile0);
        PairSync(pair);
        TV *o = a.out + e * NC;
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const int tile = tile0 + i; // rows (r = tile, q = g), n = p
            if (tile >= NM)
                break;
            double y0 = 0.0, y1 = 0.0;
            Dmma(y0, y1, c2[CubeIdx(tile, g, t)], ip0[0]);
            Dmma(y0, y1, c2[CubeIdx(tile, g, t + 4)], ip0[1]);
            if (g < NM)
            {
                if (2 * t < NM)
                    o[(tile * NM + g) * NM + 2 * t] = TV(y0);
                if (2 * t + 1 < NM)
                    o[(tile * NM + g) * NM + 2 * t + 1] = TV(y1);
            }
        }
        // the next iteration's first barrier orders these reads of c2 before
        // any later write of c2
    }
    CpAsyncWaitAll();
}

template <typename TV, int NM, bool ISO>
static int HexMma2LaunchIso(const nkb_op *op, const HexArgs<TV> &a, bool gather, cudaStream_t s,
                            bool set_attr)
{
    constexpr int NQ   = NM + 1;
    const size_t bytes = size_t(kMma2Pairs) * kMmaCubes * kMmaCube * sizeof(double);
    const int mode = HexMode(op, gather);
    if (mode < 0)
        return SetError(NKB_ERR_UNSUPPORTED, "LinearADR has no gathered Hex kernel");
    void (*kerns[3])(HexArgs<TV>, const HexConst<double, NM, NQ>) = {
        k_hex_helm_mma2<TV, NM, NQ, kModeLocal, ISO>, k_hex_helm_mma2<TV, NM, NQ, kModeGather, ISO>,
        k_hex_helm_mma2<TV, NM, NQ, kModeAdv, ISO>};
    if (set_attr)
    {
        for (auto k : kerns)
            NKB_CUDA_TRY(
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
        return NKB_OK;
    }
    if (op->nelmt == 0)
        return NKB_OK;
    static int s_per_sm[3] = {0, 0, 0}; // resident CTAs per SM of each mode
    if (s_per_sm[mode] == 0)
    {
        int b = 0;
        NKB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kerns[mode],
                                                                   64 * kMma2Pairs, bytes));
        s_per_sm[mode] = std::max(b, 1);
    }
    const long want = (long(op->nelmt) + kMma2Pairs - 1) / kMma2Pairs;
    const long nb   = std::min<long>(want, long(s_per_sm[mode]) * SmCount(op->device));
    const HexConst<double, NM, NQ> c = MakeHexConst<double, NM, NQ>(op);
    kerns[mode]<<<unsigned(nb), 64 * kMma2Pairs, bytes, s>>>(a, c);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

template <typename TV, int NM>
static int HexMma2Launch(const nkb_op *op, const HexArgs<TV> &a, bool gather, cudaStream_t s,
                         bool set_attr)
{
    if constexpr (NM + 1 > 8)
    {
        (void)op;
        (void)a;
        (void)gather;
        (void)s;
        (void)set_attr;
        return SetError(NKB_ERR_UNSUPPORTED, "the DMMA Hex kernel covers nq <= 8");
    }
    else
    {
        const bool iso = op->hB[0] == op->hB[1] && op->hB[0] == op->hB[2];
        return iso ? HexMma2LaunchIso<TV, NM, true>(op, a, gather, s, set_attr)
                   : HexMma2LaunchIso<TV, NM, false>(op, a, gather, s, set_attr);
    }
}

} // namespace nkb
