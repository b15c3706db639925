// Hex Helmholtz on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64) for
// nq <= 8. One warp per element. The arithmetic is FP64 for both operator
// precisions; an FP32 operator keeps FP32 storage (coefficients in and out,
// geometry), which halves its bytes while its rounding stays that of the
// stored data only. Every sum-factorisation contraction is a
// 64 x 8 x 8 matrix product over an 8 x 8 x 8 cube (modes and points padded
// with zeros to 8 per direction): 8 row tiles of 8 x 8 outputs, two k-steps
// of 4 each, with the 1-D table in the B fragment and the cube rows in the
// A fragment. Twelve such contractions make one element (BwdTrans 3,
// gradient 3, transposed gradient 3 accumulated in place, inner product 3),
// about 190 DMMAs; the metric step between them is pointwise. Warps are persistent
// and copy the next element's coefficients into shared memory asynchronously
// while the current one is computed; the current element's geometry is
// prefetched into L2 at the start of its turn. The arithmetic per
// element is the same fused formulation as k_hex_helm:
//   y = B^T [ lambda W u + sum_a D_a^T (G' grad u)_a ],  u = B x.
//
// Shared memory per warp: four cubes, each [c][b][a] at
// c*68 + b*8 + (a ^ 4*((b >> 1) & 1) ^ (c & 4)): the XORs on a and the
// c-stride of 68 make the A-fragment loads of all three contraction
// directions, the stores of the a- and c-contractions and the metric step's
// accesses free of bank conflicts (a 16-lane phase touches 16 distinct 8-byte
// bank pairs); the b-contraction's stores are 2-way.
//
// m8n8k4 f64 fragments (lane = 4 g + t): A (8x4, row) holds A[g][t];
// B (4x8, col) holds B[t][g]; C/D (8x8) hold C[g][2t], C[g][2t+1].
#pragma once

// included at the end of nkb_hex_kernel.cuh
#include "nkb_hex_kernel.cuh"

namespace nkb
{

constexpr int kMmaCube  = 8 * 68; // doubles per cube
constexpr int kMmaWarps = 4;      // warps per CTA (each walks its own elements)
constexpr int kMmaCubes = 4;      // shared-memory cubes per warp

__device__ __forceinline__ int CubeIdx(int c, int b, int a)
{
    return c * 68 + b * 8 + (a ^ ((b & 2) << 1) ^ (c & 4));
}

// Cubes of an FP32-storage operator hold floats (half the shared-memory
// traffic, the operator's arithmetic stays FP64): [c][b][a] at
// c*72 + b*8 + (a ^ 4*((b >> 2) & 1)), conflict-free for the A-fragment loads
// of all three directions (32 lanes, 4-byte words).
constexpr int kMmaCubeF = 8 * 72; // floats per FP32 cube

__device__ __forceinline__ int CubeIdxF(int c, int b, int a)
{
    return c * 72 + b * 8 + (a ^ (b & 4));
}

template <typename TC> __device__ __forceinline__ int CIdx(int c, int b, int a)
{
    if constexpr (sizeof(TC) == 8)
        return CubeIdx(c, b, a);
    else
        return CubeIdxF(c, b, a);
}

// elements per cube of either type
template <typename TC> constexpr int CubeLen()
{
    return sizeof(TC) == 8 ? kMmaCube : kMmaCubeF;
}

template <typename TC> struct Pair2;
template <> struct Pair2<double>
{
    using type = double2;
};
template <> struct Pair2<float>
{
    using type = float2;
};

__device__ __forceinline__ void Dmma(double &c0, double &c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// One contraction over cube axis AX (0: a, 1: b, 2: c): rows are the other two
// axes (tile = the slower, g = the faster), k and n run along AX.
// out(rows, n) (+)= sum_k in(rows, k) * B(k, n), B(k, n) in fragments bf[kk]
// (k = t + 4 kk, n = g).
template <int AX, bool ACC, typename TIN = double, typename TOUT = double>
__device__ __forceinline__ void Contract(const TIN *__restrict__ in, TOUT *__restrict__ out,
                                         const double (&bf)[2], int g, int t)
{
#pragma unroll
    for (int tile = 0; tile < 8; ++tile)
    {
        int ia0, ia1, io0, io1; // io1 = io0 + 1 when AX == 0
        if (AX == 0) // rows (c = tile, b = g)
        {
            ia0 = CIdx<TIN>(tile, g, t);
            ia1 = CIdx<TIN>(tile, g, t + 4);
            io0 = CIdx<TOUT>(tile, g, 2 * t);
            io1 = io0 + 1;
        }
        else if (AX == 1) // rows (c = tile, a = g)
        {
            ia0 = CIdx<TIN>(tile, t, g);
            ia1 = CIdx<TIN>(tile, t + 4, g);
            io0 = CIdx<TOUT>(tile, 2 * t, g);
            io1 = CIdx<TOUT>(tile, 2 * t + 1, g);
        }
        else // rows (b = tile, a = g)
        {
            ia0 = CIdx<TIN>(t, tile, g);
            ia1 = CIdx<TIN>(t + 4, tile, g);
            io0 = CIdx<TOUT>(2 * t, tile, g);
            io1 = CIdx<TOUT>(2 * t + 1, tile, g);
        }
        double c0 = 0.0, c1 = 0.0;
        if (AX == 0)
        {
            // the pair (2t, 2t+1) is adjacent and aligned: one vector access
            using P2 = typename Pair2<TOUT>::type;
            P2 *o2   = reinterpret_cast<P2 *>(out + io0);
            if (ACC)
            {
                const P2 v = *o2;
                c0         = double(v.x);
                c1         = double(v.y);
            }
            Dmma(c0, c1, double(in[ia0]), bf[0]);
            Dmma(c0, c1, double(in[ia1]), bf[1]);
            P2 w;
            w.x = TOUT(c0);
            w.y = TOUT(c1);
            *o2 = w;
        }
        else
        {
            if (ACC)
            {
                c0 = double(out[io0]);
                c1 = double(out[io1]);
            }
            Dmma(c0, c1, double(in[ia0]), bf[0]);
            Dmma(c0, c1, double(in[ia1]), bf[1]);
            out[io0] = TOUT(c0);
            out[io1] = TOUT(c1);
        }
    }
}

template <int NM, int NQ> struct MmaTabs
{
    // B fragments: modes -> points (BwdTrans) and points -> modes (inner
    // product) per direction; gradient and transposed gradient
    double bw[3][2], ip[3][2], dg[2], dt[2];
};

template <int NM, int NQ>
__device__ __forceinline__ void LoadMmaTabs(const HexConst<double, NM, NQ> &c, MmaTabs<NM, NQ> &f,
                                            int g, int t)
{
    const double *B[3] = {c.B0, c.B1, c.B2};
#pragma unroll
    for (int kk = 0; kk < 2; ++kk)
    {
        const int k = t + 4 * kk;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            // BwdTrans: B(k = mode, n = point) = phi_k(z_n)
            f.bw[d][kk] = (k < NM && g < NQ) ? B[d][k * NQ + g] : 0.0;
            // inner product: B(k = point, n = mode) = phi_n(z_k)
            f.ip[d][kk] = (g < NM && k < NQ) ? B[d][g * NQ + k] : 0.0;
        }
        // gradient: B(k = m, n = i) = l_m'(z_i) = D[i*NQ + m]
        f.dg[kk] = (g < NQ && k < NQ) ? c.D[g * NQ + k] : 0.0;
        // transposed gradient: B(k = m, n = i) = l_i'(z_m) = D[m*NQ + i]
        f.dt[kk] = (g < NQ && k < NQ) ? c.D[k * NQ + g] : 0.0;
    }
}

// Coefficients reach shared memory by asynchronous copies (cp.async, no
// registers held while they are in flight), gathered through the map, one
// element ahead; the map entries themselves are read two elements ahead.
__device__ __forceinline__ void CpAsync(double *dst, const double *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(SmemAddr(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void CpAsync(float *dst, const float *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(SmemAddr(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void CpAsyncCommit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void CpAsyncWaitAll()
{
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// map entries (or plain offsets) of element e for the lane's 16 cube positions
template <int NM, bool GATHER, typename TV>
__device__ __forceinline__ void LoadMap(const HexArgs<TV> &a, long e, int lane, int (&idx)[16])
{
    constexpr int NC = NM * NM * NM;
#pragma unroll
    for (int s = 0; s < 16; ++s)
    {
        const int pos = lane + 32 * s;
        const int cc = pos >> 6, bb = (pos >> 3) & 7, aa = pos & 7;
        const int m  = (cc * NM + bb) * NM + aa;
        const bool real = aa < NM && bb < NM && cc < NM;
        idx[s]          = real ? (GATHER ? __ldg(a.gmap + e * NC + m) : m) : -1;
    }
}

// coefficients of element e into the cube x (real positions only; the padded
// ones stay zero)
template <int NM, bool GATHER, typename TV>
__device__ __forceinline__ void FetchCoeffs(const HexArgs<TV> &a, long e, int lane,
                                            const int (&idx)[16], TV *x)
{
    constexpr int NC = NM * NM * NM;
#pragma unroll
    for (int s = 0; s < 16; ++s)
    {
        if (idx[s] < 0)
            continue;
        const int pos = lane + 32 * s;
        TV *dst       = x + CIdx<TV>(pos >> 6, (pos >> 3) & 7, pos & 7);
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

// Persistent: each warp walks the elements e = warp id, warp id + warps, ...
// Per warp four cubes in shared memory: x (coefficients, filled
// asynchronously), c0, c1, c2. The z-gradient and lambda W u never leave
// registers (the metric step runs in the C-fragment layout of the z
// contraction, which is also the layout of the first transposed-gradient
// contraction). Geometry is read with read-only loads in four batches of four
// points per lane, all loads of a batch issued before any of its stores.
template <typename TV, int NM, int NQ, int MODE>
__global__ void __launch_bounds__(32 * kMmaWarps, sizeof(TV) == 8 ? 3 : 4)
    k_hex_helm_mma(HexArgs<TV> a, const __grid_constant__ HexConst<double, NM, NQ> c)
{
    constexpr bool GATHER = MODE == kModeGather, ADV = MODE == kModeAdv;
    constexpr int NG      = ADV ? 10 : 7; // packed values per point
    static_assert(NQ <= 8 && NM < NQ, "the DMMA Hex kernel covers nq <= 8");
    constexpr int NQ2 = NQ * NQ, NQ3 = NQ2 * NQ, NC = NM * NM * NM;
    extern __shared__ __align__(16) double msm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const long nwarps = long(gridDim.x) * kMmaWarps;
    long e            = long(blockIdx.x) * kMmaWarps + warp;
    if (e >= a.nelmt || (a.skip && *a.skip))
        return;
    // cubes hold the storage type: doubles for an FP64 operator, floats for
    // an FP32-storage one (the arithmetic is FP64 either way)
    using TC        = TV;
    constexpr int CL = CubeLen<TC>();
    TC *xc = reinterpret_cast<TC *>(msm) + warp * kMmaCubes * CL; // coefficients
    TC *c0 = xc + CL, *c1 = c0 + CL, *c2 = c1 + CL;
    const uint32_t gbytes = uint32_t(NG * NQ3 * sizeof(TV) + 15) & ~15u;

    MmaTabs<NM, NQ> f;
    LoadMmaTabs<NM, NQ>(c, f, g, t);
    const double lam = double(a.lambda);

    // the padded positions of the coefficient cube stay zero for good
    for (int pos = lane; pos < CL; pos += 32)
        xc[pos] = TC(0);
    __syncwarp();
    int idx[16];
    LoadMap<NM, GATHER, TV>(a, e, lane, idx);
    FetchCoeffs<NM, GATHER, TV>(a, e, lane, idx, xc);
    if (e + nwarps < a.nelmt)
        LoadMap<NM, GATHER, TV>(a, e + nwarps, lane, idx);

    for (; e < a.nelmt; e += nwarps)
    {
        const TV *__restrict__ G = a.geo + e * a.gstride;
        // this element's geometry is read after BwdTrans and the gradient:
        // bring it into L2 now (a whole element earlier it is evicted again)
        if (lane == 0)
            BulkPrefetchL2(G, gbytes);
        CpAsyncWaitAll();
        __syncwarp();
        // BwdTrans: p -> i (x -> c1), q -> j (c1 -> c0), r -> k (c0 -> c1 = u)
        Contract<0, false>(xc, c1, f.bw[0], g, t);
        __syncwarp();
        const long en = e + nwarps;
        if (en < a.nelmt)
        {
            FetchCoeffs<NM, GATHER, TV>(a, en, lane, idx, xc); // x is free again
            if (en + nwarps < a.nelmt)
                LoadMap<NM, GATHER, TV>(a, en + nwarps, lane, idx);
        }
        Contract<1, false>(c1, c0, f.bw[1], g, t);
        __syncwarp();
        Contract<2, false>(c0, c1, f.bw[2], g, t);
        __syncwarp();
        // gradient: g0 -> c0, g1 -> c2, g2 in registers (rows (b = tile, a = g),
        // columns c = 2t, 2t + 1)
        Contract<0, false>(c1, c0, f.dg, g, t);
        Contract<1, false>(c1, c2, f.dg, g, t);
        double z[8][2];
#pragma unroll
        for (int tile = 0; tile < 8; ++tile)
        {
            z[tile][0] = z[tile][1] = 0.0;
            Dmma(z[tile][0], z[tile][1], double(c1[CIdx<TC>(t, tile, g)]), f.dg[0]);
            Dmma(z[tile][0], z[tile][1], double(c1[CIdx<TC>(t + 4, tile, g)]), f.dg[1]);
        }
        __syncwarp();
        // metric at the lane's 16 points (c = 2t + h, b = tile, a = g):
        // v0 -> c0, v1 -> c2, v2 -> c1 (over u), z <- lambda W u
#pragma unroll
        for (int tb = 0; tb < 8; tb += 2)
        {
            double gv[4][NG];
#pragma unroll
            for (int p = 0; p < 4; ++p)
            {
                const int tile = tb + (p >> 1), cc = 2 * t + (p & 1);
                const bool real = cc < NQ && tile < NQ && g < NQ;
                const int q     = real ? (cc * NQ + tile) * NQ + g : 0;
#pragma unroll
                for (int k = 0; k < NG; ++k)
                    gv[p][k] = real ? double(__ldg(G + k * NQ3 + q)) : 0.0;
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
            {
                const int tile = tb + (p >> 1), h = p & 1;
                const int ci   = CIdx<TC>(2 * t + h, tile, g);
                const double x0 = double(c0[ci]), x1 = double(c2[ci]), x2 = z[tile][h];
                const double W = gv[p][0], G00 = gv[p][1], G11 = gv[p][2], G22 = gv[p][3];
                const double G01 = gv[p][4], G02 = gv[p][5], G12 = gv[p][6];
                c0[ci]     = TC(fma(G02, x2, fma(G01, x1, G00 * x0)));
                c2[ci]     = TC(fma(G12, x2, fma(G11, x1, G01 * x0)));
                const double v2 = fma(G22, x2, fma(G12, x1, G02 * x0));
                if (ADV)
                {
                    const double adv = fma(gv[p][9 % NG], x2,
                                           fma(gv[p][8 % NG], x1, gv[p][7 % NG] * x0));
                    z[tile][h]       = lam * fma(W, double(c1[ci]), adv);
                }
                else
                {
                    z[tile][h] = lam * W * double(c1[ci]);
                }
                c1[ci]     = TC(v2);
            }
        }
        __syncwarp();
        // f = lambda W u + D_2^T v2 (registers), then + D_0^T v0 + D_1^T v1 in c1
#pragma unroll
        for (int tile = 0; tile < 8; ++tile)
        {
            Dmma(z[tile][0], z[tile][1], double(c1[CIdx<TC>(t, tile, g)]), f.dt[0]);
            Dmma(z[tile][0], z[tile][1], double(c1[CIdx<TC>(t + 4, tile, g)]), f.dt[1]);
        }
        __syncwarp();
#pragma unroll
        for (int tile = 0; tile < 8; ++tile)
        {
            c1[CIdx<TC>(2 * t, tile, g)]     = TC(z[tile][0]);
            c1[CIdx<TC>(2 * t + 1, tile, g)] = TC(z[tile][1]);
        }
        __syncwarp();
        Contract<0, true>(c0, c1, f.dt, g, t);
        __syncwarp();
        Contract<1, true>(c2, c1, f.dt, g, t);
        __syncwarp();
        // inner product: k -> r (c0), j -> q (c2), i -> p (to global)
        Contract<2, false>(c1, c0, f.ip[2], g, t);
        __syncwarp();
        Contract<1, false>(c0, c2, f.ip[1], g, t);
        __syncwarp();
        TV *o = a.out + e * NC;
#pragma unroll
        for (int tile = 0; tile < NM; ++tile) // rows (r = tile, q = g), n = p
        {
            double y0 = 0.0, y1 = 0.0;
            Dmma(y0, y1, double(c2[CIdx<TC>(tile, g, t)]), f.ip[0][0]);
            Dmma(y0, y1, double(c2[CIdx<TC>(tile, g, t + 4)]), f.ip[0][1]);
            if (g < NM)
            {
                if (2 * t < NM)
                    o[(tile * NM + g) * NM + 2 * t] = TV(y0);
                if (2 * t + 1 < NM)
                    o[(tile * NM + g) * NM + 2 * t + 1] = TV(y1);
            }
        }
    }
    CpAsyncWaitAll(); // nothing may still be copying into shared memory at exit
}

int SmCount(int device); // multiprocessors of a device (nkb_hex.cu)

template <typename TV, int NM>
static int HexMmaLaunch(const nkb_op *op, const HexArgs<TV> &a, bool gather, cudaStream_t s,
                        bool set_attr)
{
    constexpr int NQ   = NM + 1;
    const size_t bytes = size_t(kMmaWarps) * kMmaCubes * CubeLen<TV>() * sizeof(TV);
    if constexpr (NQ > 8)
    {
        (void)op;
        (void)a;
        (void)gather;
        (void)s;
        (void)set_attr;
        (void)bytes;
        return SetError(NKB_ERR_UNSUPPORTED, "the DMMA Hex kernel covers nq <= 8");
    }
    else
    {
        const int mode = HexMode(op, gather);
        if (mode < 0)
            return SetError(NKB_ERR_UNSUPPORTED, "LinearADR has no gathered Hex kernel");
        void (*kerns[3])(HexArgs<TV>, const HexConst<double, NM, NQ>) = {
            k_hex_helm_mma<TV, NM, NQ, kModeLocal>, k_hex_helm_mma<TV, NM, NQ, kModeGather>,
            k_hex_helm_mma<TV, NM, NQ, kModeAdv>};
        if (set_attr)
        {
            for (auto k : kerns)
                NKB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  int(bytes)));
            return NKB_OK;
        }
        if (op->nelmt == 0)
            return NKB_OK;
        // persistent grid: as many CTAs as stay resident, fewer for small operators
        static int s_per_sm[3] = {0, 0, 0}; // resident CTAs per SM of each mode
        if (s_per_sm[mode] == 0)
        {
            int b = 0;
            NKB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kerns[mode],
                                                                       32 * kMmaWarps, bytes));
            s_per_sm[mode] = std::max(b, 1);
        }
        const long want = (long(op->nelmt) + kMmaWarps - 1) / kMmaWarps;
        const long nb   = std::min<long>(want, long(s_per_sm[mode]) * SmCount(op->device));
        const HexConst<double, NM, NQ> c = MakeHexConst<double, NM, NQ>(op);
        kerns[mode]<<<unsigned(nb), 32 * kMmaWarps, bytes, s>>>(a, c);
        NKB_CUDA_TRY(cudaGetLastError());
        return NKB_OK;
    }
}

} // namespace nkb

#include "nkb_hex_mma2.cuh"
