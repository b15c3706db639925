// Hex Helmholtz on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64) for
// nq <= 8. One warp per element. Every sum-factorisation contraction is a
// 64 x 8 x 8 matrix product over an 8 x 8 x 8 cube (modes and points padded
// with zeros to 8 per direction): 8 row tiles of 8 x 8 outputs, two k-steps
// of 4 each, with the 1-D table in the B fragment and the cube rows in the
// A fragment. Twelve such contractions make one element (BwdTrans 3,
// gradient 3, transposed gradient 3 accumulated in place, inner product 3),
// 192 DMMAs; the metric step between them is pointwise. The arithmetic per
// element is the same fused formulation as k_hex_helm:
//   y = B^T [ lambda W u + sum_a D_a^T (G' grad u)_a ],  u = B x.
//
// Shared memory per warp: four cubes, each [c][b][a] at
// c*68 + b*8 + (a ^ 4*((b >> 1) & 1)): the XOR on a and the c-stride of 68
// make the A-fragment loads of all three contraction directions free of bank
// conflicts (a 16-lane phase touches 16 distinct 8-byte bank pairs).
//
// m8n8k4 f64 fragments (lane = 4 g + t): A (8x4, row) holds A[g][t];
// B (4x8, col) holds B[t][g]; C/D (8x8) hold C[g][2t], C[g][2t+1].
#pragma once

// included at the end of nkb_hex_kernel.cuh
#include "nkb_hex_kernel.cuh"

namespace nkb
{

constexpr int kMmaCube  = 8 * 68; // doubles per cube
constexpr int kMmaWarps = 4;      // warps (elements) per CTA

__device__ __forceinline__ int CubeIdx(int c, int b, int a)
{
    return c * 68 + b * 8 + (a ^ ((b & 2) << 1));
}

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
template <int AX, bool ACC>
__device__ __forceinline__ void Contract(const double *__restrict__ in, double *__restrict__ out,
                                         const double (&bf)[2], int g, int t)
{
#pragma unroll
    for (int tile = 0; tile < 8; ++tile)
    {
        int ia0, ia1, io0, io1;
        if (AX == 0) // rows (c = tile, b = g)
        {
            ia0 = CubeIdx(tile, g, t);
            ia1 = CubeIdx(tile, g, t + 4);
            io0 = CubeIdx(tile, g, 2 * t);
            io1 = CubeIdx(tile, g, 2 * t + 1);
        }
        else if (AX == 1) // rows (c = tile, a = g)
        {
            ia0 = CubeIdx(tile, t, g);
            ia1 = CubeIdx(tile, t + 4, g);
            io0 = CubeIdx(tile, 2 * t, g);
            io1 = CubeIdx(tile, 2 * t + 1, g);
        }
        else // rows (b = tile, a = g)
        {
            ia0 = CubeIdx(t, tile, g);
            ia1 = CubeIdx(t + 4, tile, g);
            io0 = CubeIdx(2 * t, tile, g);
            io1 = CubeIdx(2 * t + 1, tile, g);
        }
        double c0 = 0.0, c1 = 0.0;
        if (ACC)
        {
            c0 = out[io0];
            c1 = out[io1];
        }
        Dmma(c0, c1, in[ia0], bf[0]);
        Dmma(c0, c1, in[ia1], bf[1]);
        out[io0] = c0;
        out[io1] = c1;
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

template <int NM, int NQ, bool GATHER>
__global__ void __launch_bounds__(32 * kMmaWarps)
    k_hex_helm_mma(HexArgs<double> a, const __grid_constant__ HexConst<double, NM, NQ> c)
{
    static_assert(NQ <= 8 && NM < NQ, "the DMMA Hex kernel covers nq <= 8");
    constexpr int NQ2 = NQ * NQ, NQ3 = NQ2 * NQ, NC = NM * NM * NM;
    extern __shared__ __align__(16) double msm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const long e = long(blockIdx.x) * kMmaWarps + warp;
    if (e >= a.nelmt || (a.skip && *a.skip))
        return;
    double *c0 = msm + warp * 4 * kMmaCube, *c1 = c0 + kMmaCube, *c2 = c1 + kMmaCube,
           *c3 = c2 + kMmaCube;
    const double *G = a.geo + e * a.gstride;
    // the element's geometry is needed only after BwdTrans and the gradient:
    // start bringing it into L2 now
    if (lane == 0)
        BulkPrefetchL2(G, uint32_t(7 * NQ3 * sizeof(double) + 15) & ~15u);

    MmaTabs<NM, NQ> f;
    LoadMmaTabs<NM, NQ>(c, f, g, t);

    // coefficients into cube 0 ([r][q][p], zero padded)
#pragma unroll 4
    for (int pos = lane; pos < 512; pos += 32)
    {
        const int cc = pos >> 6, bb = (pos >> 3) & 7, aa = pos & 7;
        double v = 0.0;
        if (aa < NM && bb < NM && cc < NM)
        {
            const long gi = e * NC + (cc * NM + bb) * NM + aa;
            if (GATHER)
            {
                v = a.in[a.gmap[gi]];
                if (a.gsign)
                    v *= a.gsign[gi];
            }
            else
            {
                v = a.in[gi];
            }
        }
        c0[CubeIdx(cc, bb, aa)] = v;
    }
    __syncwarp();
    // BwdTrans: p -> i, q -> j, r -> k; u in cube 1
    Contract<0, false>(c0, c1, f.bw[0], g, t);
    __syncwarp();
    Contract<1, false>(c1, c0, f.bw[1], g, t);
    __syncwarp();
    Contract<2, false>(c0, c1, f.bw[2], g, t);
    __syncwarp();
    // reference-space gradient: g0 -> cube 0, g1 -> cube 2, g2 -> cube 3
    Contract<0, false>(c1, c0, f.dg, g, t);
    Contract<1, false>(c1, c2, f.dg, g, t);
    Contract<2, false>(c1, c3, f.dg, g, t);
    __syncwarp();
    // metric: v = G' grad u in place of the gradients, f = lambda W u in place of u
    const double lam = a.lambda;
#pragma unroll 2
    for (int q = lane; q < NQ3; q += 32)
    {
        const int kk = q / NQ2, jj = (q / NQ) % NQ, ii = q % NQ;
        const int ci = CubeIdx(kk, jj, ii);
        const double W = G[q], G00 = G[NQ3 + q], G11 = G[2 * NQ3 + q], G22 = G[3 * NQ3 + q];
        const double G01 = G[4 * NQ3 + q], G02 = G[5 * NQ3 + q], G12 = G[6 * NQ3 + q];
        const double x0 = c0[ci], x1 = c2[ci], x2 = c3[ci];
        c0[ci] = fma(G02, x2, fma(G01, x1, G00 * x0));
        c2[ci] = fma(G12, x2, fma(G11, x1, G01 * x0));
        c3[ci] = fma(G22, x2, fma(G12, x1, G02 * x0));
        c1[ci] = lam * W * c1[ci];
    }
    __syncwarp();
    // f += D_0^T v0 + D_1^T v1 + D_2^T v2 (in place, one direction at a time)
    Contract<0, true>(c0, c1, f.dt, g, t);
    __syncwarp();
    Contract<1, true>(c2, c1, f.dt, g, t);
    __syncwarp();
    Contract<2, true>(c3, c1, f.dt, g, t);
    __syncwarp();
    // inner product: k -> r (cube 0), j -> q (cube 2), i -> p (to global)
    Contract<2, false>(c1, c0, f.ip[2], g, t);
    __syncwarp();
    Contract<1, false>(c0, c2, f.ip[1], g, t);
    __syncwarp();
    double *o = a.out + e * NC;
#pragma unroll
    for (int tile = 0; tile < NM; ++tile) // rows (r = tile, q = g), n = p
    {
        double y0 = 0.0, y1 = 0.0;
        Dmma(y0, y1, c2[CubeIdx(tile, g, t)], f.ip[0][0]);
        Dmma(y0, y1, c2[CubeIdx(tile, g, t + 4)], f.ip[0][1]);
        if (g < NM)
        {
            if (2 * t < NM)
                o[(tile * NM + g) * NM + 2 * t] = y0;
            if (2 * t + 1 < NM)
                o[(tile * NM + g) * NM + 2 * t + 1] = y1;
        }
    }
}

template <int NM>
static int HexMmaLaunch(const nkb_op *op, const HexArgs<double> &a, bool gather, cudaStream_t s,
                        bool set_attr)
{
    constexpr int NQ   = NM + 1;
    const size_t bytes = size_t(kMmaWarps) * 4 * kMmaCube * sizeof(double);
    if constexpr (NQ > 8)
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
        if (set_attr)
        {
            NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm_mma<NM, NQ, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(bytes)));
            NKB_CUDA_TRY(cudaFuncSetAttribute(k_hex_helm_mma<NM, NQ, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(bytes)));
            return NKB_OK;
        }
        const long nb = (long(op->nelmt) + kMmaWarps - 1) / kMmaWarps;
        if (nb == 0)
            return NKB_OK;
        const HexConst<double, NM, NQ> c = MakeHexConst<double, NM, NQ>(op);
        if (gather)
            k_hex_helm_mma<NM, NQ, true><<<unsigned(nb), 32 * kMmaWarps, bytes, s>>>(a, c);
        else
            k_hex_helm_mma<NM, NQ, false><<<unsigned(nb), 32 * kMmaWarps, bytes, s>>>(a, c);
        NKB_CUDA_TRY(cudaGetLastError());
        return NKB_OK;
    }
}

} // namespace nkb
