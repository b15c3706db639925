// Hex Helmholtz on the fifth-generation tensor cores (tcgen05, TF32 operands
// split into high and low parts, FP32 accumulation in tensor memory): the
// FP32 inner operator of the mixed-precision CG.
//
// The element operator of MatrixFreeOps/Helmholtz.h:549-599 (fusedKernel3D)
// written as six batched contractions over M = 128 row tiles (EPT elements
// of RPE rows each), with the derivative basis dB = D B (Basis.cpp:493-495)
// so that u and its three reference derivatives come out of the same
// contractions and land in the same thread:
//
//   1  p -> i   x           x [B0 | dB0]        -> T, T'        rows (r, q)
//   2  q -> j   T, T'       x [B1 | dB1], B1    -> U, U', V     rows (r, i)
//   3  r -> k   U, U', V    x [B2 | dB2], B2    -> u, d2, d1, d0 rows (i, j)
//      metric   f = lambda W u, v = G' (d0, d1, d2)            (registers)
//   4  k -> r   f B2 + v2 dB2, v1 B2, v0 B2     -> X, Y1, Y0    rows (i, j)
//   5  j -> q   X B1 + Y1 dB1, Y0 B1            -> Z, Z0        rows (i, r)
//   6  i -> p   Z B0 + Z0 dB0                   -> y            rows (r, q)
//
// Each stage: every thread writes its values into the next stage's A
// operands in shared memory, all K-major (TF32 MMAs read MN-major operands
// as zeros on sm_100a: measured with every no-swizzle layout and stride
// assignment tried), as 16-byte rows when the thread holds the contracted
// index and as bank-spread scalar columns when it holds the rows; one thread
// issues the MMAs (A high and low parts against [B_hi | B_lo]), commits them
// to an mbarrier, and each thread reads its tensor-memory lane back and adds
// the two halves. Tables:
// for direction d, [B_hi | B_lo | dB_hi | dB_lo] with the contracted index as
// K (host-built, nkb_hex.cu BuildTcTables). One warpgroup per CTA, one row
// per thread. All waits are bounded; the tensor memory is freed on every path.
#pragma once

#include "nkb_tc.cuh"
#include "nkb_tma.cuh"

#include <type_traits>

namespace nkb
{

template <int NM, int NQ> struct TcDims
{
    static constexpr int Pad8(int v) { return (v + 7) / 8 * 8; }
    static constexpr int Pad4(int v) { return (v + 3) / 4 * 4; }
    static constexpr int Max(int x, int y) { return x > y ? x : y; }
    static constexpr int KM = Pad8(NM), KQ = Pad8(NQ);
    static constexpr int KSM = KM / 8, KSQ = KQ / 8, KS = Max(KSM, KSQ);
    static constexpr int NQP = Pad8(NQ), NMN = Pad8(NM);
    // nq <= 8: row strides of 8 and the padded operand layout, so a column
    // store's offset is a compile-time constant from its row group; larger
    // orders: strides of 4 (128 rows hold one element) and rotated stores
    static constexpr bool FAST = NQ <= 8;
    using AL                   = typename std::conditional<FAST, tc::ALayoutPad, tc::ALayoutStd>::type;
    static constexpr int QP = FAST ? 8 : Pad4(NQ), MP = FAST ? 8 : Pad4(NM);
    static constexpr int RPE0 = Max(Max(NM * MP, NM * QP), Max(NQ * QP, NQ * MP));
    static constexpr int RPE  = FAST ? Pad8(RPE0) : Pad4(RPE0);
    static constexpr int EPT   = 128 / RPE;
    static constexpr int NCUBE = 4;             // operands of the widest stage
    static constexpr int CUBE  = KS * AL::STEP; // bytes of one high or low part
    static constexpr int ABYTES = 2 * NCUBE * CUBE;
    static constexpr int TCOLS  = 8 * NQP <= 64 ? 64 : (8 * NQP <= 128 ? 128 : 256);
    static constexpr int TBROWS = 4 * NQP, TBTROWS = 4 * NMN;
    static constexpr int TB_BYTES = TBROWS * KM * 4, TBT_BYTES = TBTROWS * KQ * 4;
    // CTAs per SM that shared memory (with the tables of one direction: Hex
    // directions share their tables) and tensor memory (512 columns) allow;
    // the launch bounds ask for that many
    static constexpr int SMEM_CTAS = (227 * 1024) / (ABYTES + TB_BYTES + TBT_BYTES + 16);
    static constexpr int MIN_CTAS  = SMEM_CTAS < 512 / TCOLS ? SMEM_CTAS : 512 / TCOLS;
    static_assert(RPE <= 128, "tensor-core Hex kernel: element rows exceed one 128-row tile");
    static_assert(NQP == 8 || NQP == 16, "tensor-core Hex kernel: nq up to 16");
};

// the tensor-core kernel covers nm = 2..9 with nq = nm + 1
constexpr int kTcMinNm = 2, kTcMaxNm = 9;

struct TcTables
{
    const float *tab; // global image of the shared-memory tables
    int bytes;        // multiple of 128
    int tb[3];        // byte offset of direction d's coefficient -> point table
    int tbt[3];       // ... and of its point -> coefficient table
};

template <int NM, int NQ> constexpr size_t TcSmemBytes(int tab_bytes)
{
    return size_t(tab_bytes) + size_t(TcDims<NM, NQ>::ABYTES) + 16;
}

namespace tcd
{
// high / low parts of four values
__device__ __forceinline__ void Split4(const float *v, float4 &hi, float4 &lo)
{
    hi.x = tc::Tf32Hi(v[0]);
    hi.y = tc::Tf32Hi(v[1]);
    hi.z = tc::Tf32Hi(v[2]);
    hi.w = tc::Tf32Hi(v[3]);
    lo.x = v[0] - hi.x;
    lo.y = v[1] - hi.y;
    lo.z = v[2] - hi.z;
    lo.w = v[3] - hi.w;
}

// row m of a K-major operand pair (layout L): values v[0, LEN), zero up to KPAD
template <class L, int LEN, int KPAD>
__device__ __forceinline__ void WriteRowK(unsigned char *hi, unsigned char *lo, int m, const float *v)
{
#pragma unroll
    for (int c = 0; c < KPAD / 4; ++c)
    {
        float w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            w[u] = (4 * c + u < LEN) ? v[4 * c + u] : 0.f;
        float4 h, l;
        Split4(w, h, l);
        const uint32_t o = L::Off(m, 4 * c);
        *reinterpret_cast<float4 *>(hi + o) = h;
        *reinterpret_cast<float4 *>(lo + o) = l;
    }
}

// rows m0 .. m0 + LEN - 1 of K column k of a K-major operand pair (a thread
// that holds one K index of many rows): scalar stores.
// ROT = false (m0 % 8 == 0, padded layout): offsets from the first store are
// compile-time constants; the layout spreads a warp's stores over the banks.
// ROT = true: the stores are visited in the order starting at row m0 + s
// (s < LEN) so that the threads of a warp, given distinct s where they share
// k % 4, hit distinct banks (the bank of element (m, k) is (m % 8) * 4 + k % 4
// in the standard layout); the value array is rotated with compile-time
// indices (selects), keeping it in registers.
template <class L, int LEN, bool ROT>
__device__ __forceinline__ void WriteColK(unsigned char *hi, unsigned char *lo, int m0, int k,
                                          const float *v, int s)
{
    if constexpr (!ROT)
    {
        const uint32_t base = L::Off(m0, k);
#pragma unroll
        for (int c = 0; c < LEN; ++c)
        {
            const float h    = tc::Tf32Hi(v[c]);
            const uint32_t o = base + uint32_t(c >> 3) * uint32_t(L::SBO) + uint32_t(c & 7) * 16u;
            *reinterpret_cast<float *>(hi + o) = h;
            *reinterpret_cast<float *>(lo + o) = v[c] - h;
        }
    }
    else
    {
        float w[LEN];
#pragma unroll
        for (int j = 0; j < LEN; ++j)
            w[j] = v[j];
#pragma unroll
        for (int bit = 1; bit < LEN; bit <<= 1)
        {
            const bool on = (s & bit) != 0;
            float r[LEN];
#pragma unroll
            for (int j = 0; j < LEN; ++j)
                r[j] = w[(j + bit) % LEN];
#pragma unroll
            for (int j = 0; j < LEN; ++j)
                w[j] = on ? r[j] : w[j];
        }
#pragma unroll
        for (int j = 0; j < LEN; ++j)
        {
            int c = s + j;
            c     = c >= LEN ? c - LEN : c;
            const float h = tc::Tf32Hi(w[j]);
            const uint32_t o = L::Off(m0 + c, k);
            *reinterpret_cast<float *>(hi + o) = h;
            *reinterpret_cast<float *>(lo + o) = w[j] - h;
        }
    }
}

// sum of the high and low halves of NP + NP tensor-memory columns at taddr
template <int NP> __device__ __forceinline__ void LdPair(uint32_t taddr, float *out)
{
    static_assert(NP == 8 || NP == 16, "column pair width");
    if constexpr (NP == 8)
    {
        uint32_t r[16];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
                     "%9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
                     "tcgen05.wait::ld.sync.aligned;"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                       "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                       "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                     : "r"(taddr)
                     : "memory");
#pragma unroll
        for (int i = 0; i < 8; ++i)
            out[i] = __uint_as_float(r[i]) + __uint_as_float(r[8 + i]);
    }
    else
    {
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            uint32_t r[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, "
                         "[%16];\n\t"
                         "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8, %9, %10, %11, %12, %13, %14, "
                         "%15}, [%17];\n\t"
                         "tcgen05.wait::ld.sync.aligned;"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                           "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
                           "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                         : "r"(taddr + 8 * h), "r"(taddr + 16 + 8 * h)
                         : "memory");
#pragma unroll
            for (int i = 0; i < 8; ++i)
                out[8 * h + i] = __uint_as_float(r[i]) + __uint_as_float(r[8 + i]);
        }
    }
}

// MMAs of one K-major operand pair of layout L (high part at a_hi, low part
// a_hi + cube) against rows [n0, n0 + n) of a B table of nrows rows at stab,
// over ks K steps, into tensor-memory column tcol (acc: add to what is there)
template <class L>
__device__ __forceinline__ void IssuePair(uint32_t a_hi, uint32_t cube, uint32_t stab, int nrows,
                                          int n0, int n, int ks, uint32_t tcol, bool acc)
{
    const uint32_t idesc = tc::IDescTf32(n);
    for (int s = 0; s < ks; ++s)
    {
        const uint64_t b = tc::DescKMajor(stab + uint32_t(s * nrows * 32 + (n0 >> 3) * 256));
        const uint32_t ah = a_hi + uint32_t(s) * uint32_t(L::STEP);
        const uint32_t al = ah + cube;
        const uint64_t dh = tc::Desc(ah, L::LBO, L::SBO);
        const uint64_t dl = tc::Desc(al, L::LBO, L::SBO);
        tc::MmaTf32(tcol, dh, b, idesc, acc || s > 0);
        tc::MmaTf32(tcol, dl, b, idesc, true);
    }
}
} // namespace tcd

template <int NM, int NQ, int MODE>
__global__ void __launch_bounds__(128, TcDims<NM, NQ>::MIN_CTAS)
    k_hex_helm_tc(HexArgs<float> a, TcTables tt)
{
    using Dm = TcDims<NM, NQ>;
    constexpr int NC = NM * NM * NM, NQ2 = NQ * NQ, NT = NQ2 * NQ;
    constexpr int RPE = Dm::RPE, EPT = Dm::EPT, MP = Dm::MP, QP = Dm::QP;
    constexpr int NQP = Dm::NQP, NMN = Dm::NMN, CUBE = Dm::CUBE;
    using AL          = typename Dm::AL;
    extern __shared__ __align__(1024) unsigned char sm[];
    if (a.skip && *a.skip)
        return;
    const int t = threadIdx.x, warp = t >> 5;
    unsigned char *abuf = sm + tt.bytes;
    uint64_t *bar       = reinterpret_cast<uint64_t *>(abuf + Dm::ABYTES);
    uint32_t *slot      = reinterpret_cast<uint32_t *>(bar + 1);

    const long ntiles = (long(a.nelmt) + EPT - 1) / EPT;
    // geometry of a tile into L2 (read at the metric step)
    auto prefetch_geo = [&](long tile) {
        if (t == 0 && tile < ntiles)
        {
            const long e0 = tile * EPT;
            const long ne = (a.nelmt - e0) < EPT ? (a.nelmt - e0) : EPT;
            BulkPrefetchL2(a.geo + e0 * a.gstride, uint32_t(ne * a.gstride * sizeof(float)));
        }
    };
    prefetch_geo(blockIdx.x);
    for (int o = t * 16; o < tt.bytes; o += 128 * 16)
        *reinterpret_cast<float4 *>(sm + o) =
            __ldg(reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(tt.tab) + o));
    for (int o = t * 16; o < Dm::ABYTES; o += 128 * 16)
        *reinterpret_cast<float4 *>(abuf + o) = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t == 0)
        MbarInit(bar, 1);
    if (warp == 0)
        tc::Alloc(slot, Dm::TCOLS);
    tc::FenceProxyAsync();
    tc::FenceBeforeSync();
    __syncthreads();
    tc::FenceAfterSync();
    const uint32_t tmem = *slot;
    const uint32_t tl   = tmem + (uint32_t((warp & 3) * 32) << 16); // this warp's lanes
    const uint32_t sa   = tc::SmemU32(abuf);
    const uint32_t st   = tc::SmemU32(sm);

    const int e    = t / RPE, rr = t % RPE;
    const int rowb = e * RPE; // first row of this thread's element in a tile
    bool ok        = true;
    uint32_t phase = 0;
    const unsigned polls = WaitPolls(a.err);
    auto cube_hi = [&](int c) { return abuf + 2 * c * CUBE; };
    auto cube_lo = [&](int c) { return abuf + (2 * c + 1) * CUBE; };
    auto sync_issue = [&]() {
        tc::FenceProxyAsync();
        tc::FenceBeforeSync();
        __syncthreads();
    };
    auto wait_mma = [&]() {
        ok = MbarWaitBounded(bar, phase, a.err, 2, polls) && ok;
        phase ^= 1u;
        tc::FenceAfterSync();
    };
    const uint32_t ccube = uint32_t(CUBE);
    auto ahi = [&](int c) { return sa + uint32_t(2 * c * CUBE); };
    // this thread's coefficient row (r, q) of a tile's element: its nm values
    const int xr = rr / MP, xq = rr % MP;
    auto load_x = [&](long tile, float *x) {
        const long el = tile * EPT + e;
        if (!(tile < ntiles && e < EPT && el < a.nelmt && xr < NM && xq < NM))
            return;
        const long l0 = el * NC + (xr * NM + xq) * NM;
#pragma unroll
        for (int p = 0; p < NM; ++p)
        {
            if (MODE == kModeGather)
            {
                const int gi = a.gmap[l0 + p];
                x[p]         = a.gsign ? float(a.gsign[l0 + p]) * a.in[gi] : a.in[gi];
            }
            else
                x[p] = a.in[l0 + p];
        }
    };
    float xcur[NM];
#pragma unroll
    for (int p = 0; p < NM; ++p)
        xcur[p] = 0.f;
    load_x(blockIdx.x, xcur);

    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
    const long elem = tile * EPT + e;
    const bool ev   = e < EPT && elem < a.nelmt;
    prefetch_geo(tile + gridDim.x);

    // ---- stage 1: contract p (rows (r, q), K-major) ----------------------
    if (ev && xr < NM && xq < NM)
        tcd::WriteRowK<AL, NM, Dm::KM>(cube_hi(0), cube_lo(0), t, xcur);
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        tcd::IssuePair<AL>(ahi(0), ccube, st + tt.tb[0], Dm::TBROWS, 0, 4 * NQP, Dm::KSM, tmem,
                       false);
        tc::Commit(bar);
    }
    wait_mma();
    float T[NQP], Tp[NQP];
    tcd::LdPair<NQP>(tl, T);
    tcd::LdPair<NQP>(tl + 2 * NQP, Tp);

    // ---- stage 2: contract q (rows (r, i); this thread holds column q) -----
    {
        const int r = rr / MP, q = rr % MP;
        if (ev && r < NM && q < NM)
        {
            const int sr = (rr >> 2) % NQ; // distinct where q % 4 is shared
            tcd::WriteColK<AL, NQ, !Dm::FAST>(cube_hi(0), cube_lo(0), rowb + r * QP, q, T, sr);
            tcd::WriteColK<AL, NQ, !Dm::FAST>(cube_hi(1), cube_lo(1), rowb + r * QP, q, Tp, sr);
        }
    }
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        tcd::IssuePair<AL>(ahi(0), ccube, st + tt.tb[1], Dm::TBROWS, 0, 4 * NQP, Dm::KSM, tmem,
                       false);
        tcd::IssuePair<AL>(ahi(1), ccube, st + tt.tb[1], Dm::TBROWS, 0, 2 * NQP, Dm::KSM,
                       tmem + 4 * NQP, false);
        tc::Commit(bar);
    }
    wait_mma();
    float U[NQP], Up[NQP], V[NQP];
    tcd::LdPair<NQP>(tl, U);
    tcd::LdPair<NQP>(tl + 2 * NQP, Up);
    tcd::LdPair<NQP>(tl + 4 * NQP, V);

    // ---- stage 3: contract r (rows (i, j); this thread holds column r) -----
    {
        const int r = rr / QP, i = rr % QP;
        if (ev && r < NM && i < NQ)
        {
            const int sr = i % NQ; // distinct where r % 4 is shared
            tcd::WriteColK<AL, NQ, !Dm::FAST>(cube_hi(0), cube_lo(0), rowb + i * QP, r, U, sr);
            tcd::WriteColK<AL, NQ, !Dm::FAST>(cube_hi(1), cube_lo(1), rowb + i * QP, r, Up, sr);
            tcd::WriteColK<AL, NQ, !Dm::FAST>(cube_hi(2), cube_lo(2), rowb + i * QP, r, V, sr);
        }
    }
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        tcd::IssuePair<AL>(ahi(0), ccube, st + tt.tb[2], Dm::TBROWS, 0, 4 * NQP, Dm::KSM, tmem,
                       false);
        tcd::IssuePair<AL>(ahi(1), ccube, st + tt.tb[2], Dm::TBROWS, 0, 2 * NQP, Dm::KSM,
                       tmem + 4 * NQP, false);
        tcd::IssuePair<AL>(ahi(2), ccube, st + tt.tb[2], Dm::TBROWS, 0, 2 * NQP, Dm::KSM,
                       tmem + 6 * NQP, false);
        tc::Commit(bar);
    }
    wait_mma();
    // u, d2 (from U), d1 (U'), d0 (V) at this thread's point column (i, j)
    float u[NQP], g2[NQP], g1[NQP], g0[NQP];
    tcd::LdPair<NQP>(tl, u);
    tcd::LdPair<NQP>(tl + 2 * NQP, g2);
    tcd::LdPair<NQP>(tl + 4 * NQP, g1);
    tcd::LdPair<NQP>(tl + 6 * NQP, g0);

    // ---- metric, then stage 4: contract k (rows (i, j), K-major) -----------
    {
        const int i = rr / QP, j = rr % QP;
        if (ev && i < NQ && j < NQ)
        {
            const float *G = a.geo + elem * a.gstride + j * NQ + i;
            const float lam = a.lambda;
            float f[NQ], v0[NQ], v1[NQ], v2[NQ];
#pragma unroll
            for (int k = 0; k < NQ; ++k)
            {
                const int q     = k * NQ2;
                const float W   = __ldg(G + q);
                const float G00 = __ldg(G + NT + q), G11 = __ldg(G + 2 * NT + q);
                const float G22 = __ldg(G + 3 * NT + q), G01 = __ldg(G + 4 * NT + q);
                const float G02 = __ldg(G + 5 * NT + q), G12 = __ldg(G + 6 * NT + q);
                f[k]  = lam * W * u[k];
                v0[k] = fmaf(G02, g2[k], fmaf(G01, g1[k], G00 * g0[k]));
                v1[k] = fmaf(G12, g2[k], fmaf(G11, g1[k], G01 * g0[k]));
                v2[k] = fmaf(G22, g2[k], fmaf(G12, g1[k], G02 * g0[k]));
            }
            tcd::WriteRowK<AL, NQ, Dm::KQ>(cube_hi(0), cube_lo(0), t, f);
            tcd::WriteRowK<AL, NQ, Dm::KQ>(cube_hi(1), cube_lo(1), t, v2);
            tcd::WriteRowK<AL, NQ, Dm::KQ>(cube_hi(2), cube_lo(2), t, v1);
            tcd::WriteRowK<AL, NQ, Dm::KQ>(cube_hi(3), cube_lo(3), t, v0);
        }
    }
    // the next tile's coefficients, in flight during the last three stages
    load_x(tile + gridDim.x, xcur);
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        const uint32_t tb = st + tt.tbt[2];
        tcd::IssuePair<AL>(ahi(0), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem, false);
        tcd::IssuePair<AL>(ahi(1), ccube, tb, Dm::TBTROWS, 2 * NMN, 2 * NMN, Dm::KSQ, tmem, true);
        tcd::IssuePair<AL>(ahi(2), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem + 2 * NMN,
                       false);
        tcd::IssuePair<AL>(ahi(3), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem + 4 * NMN,
                       false);
        tc::Commit(bar);
    }
    wait_mma();
    float X[NMN], Y1[NMN], Y0[NMN];
    tcd::LdPair<NMN>(tl, X);
    tcd::LdPair<NMN>(tl + 2 * NMN, Y1);
    tcd::LdPair<NMN>(tl + 4 * NMN, Y0);

    // ---- stage 5: contract j (rows (i, r); this thread holds column j) -----
    {
        const int i = rr / QP, j = rr % QP;
        if (ev && i < NQ && j < NQ)
        {
            const int sr = (rr >> 2) % NM; // distinct where j % 4 is shared
            tcd::WriteColK<AL, NM, !Dm::FAST>(cube_hi(0), cube_lo(0), rowb + i * MP, j, X, sr);
            tcd::WriteColK<AL, NM, !Dm::FAST>(cube_hi(1), cube_lo(1), rowb + i * MP, j, Y1, sr);
            tcd::WriteColK<AL, NM, !Dm::FAST>(cube_hi(2), cube_lo(2), rowb + i * MP, j, Y0, sr);
        }
    }
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        const uint32_t tb = st + tt.tbt[1];
        tcd::IssuePair<AL>(ahi(0), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem, false);
        tcd::IssuePair<AL>(ahi(1), ccube, tb, Dm::TBTROWS, 2 * NMN, 2 * NMN, Dm::KSQ, tmem, true);
        tcd::IssuePair<AL>(ahi(2), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem + 2 * NMN,
                       false);
        tc::Commit(bar);
    }
    wait_mma();
    float Z[NMN], Z0[NMN];
    tcd::LdPair<NMN>(tl, Z);
    tcd::LdPair<NMN>(tl + 2 * NMN, Z0);

    // ---- stage 6: contract i (rows (r, q); this thread holds column i) -----
    {
        const int i = rr / MP, r = rr % MP;
        if (ev && i < NQ && r < NM)
        {
            const int sr = r % NM; // distinct where i % 4 is shared
            tcd::WriteColK<AL, NM, !Dm::FAST>(cube_hi(0), cube_lo(0), rowb + r * MP, i, Z, sr);
            tcd::WriteColK<AL, NM, !Dm::FAST>(cube_hi(1), cube_lo(1), rowb + r * MP, i, Z0, sr);
        }
    }
    sync_issue();
    if (t == 0)
    {
        tc::FenceAfterSync();
        const uint32_t tb = st + tt.tbt[0];
        tcd::IssuePair<AL>(ahi(0), ccube, tb, Dm::TBTROWS, 0, 2 * NMN, Dm::KSQ, tmem, false);
        tcd::IssuePair<AL>(ahi(1), ccube, tb, Dm::TBTROWS, 2 * NMN, 2 * NMN, Dm::KSQ, tmem, true);
        tc::Commit(bar);
    }
    wait_mma();
    float y[NMN];
    tcd::LdPair<NMN>(tl, y);
    {
        const int r = rr / MP, q = rr % MP;
        if (ok && ev && r < NM && q < NM)
        {
            float *o = a.out + elem * NC + (r * NM + q) * NM;
#pragma unroll
            for (int p = 0; p < NM; ++p)
                o[p] = y[p];
        }
    }

    }

    // every tensor-memory read and every MMA is complete here
    tc::FenceBeforeSync();
    __syncthreads();
    if (warp == 0)
    {
        tc::FenceAfterSync();
        tc::Dealloc(tmem, Dm::TCOLS);
    }
    if (t == 0)
        MbarInval(bar);
}

} // namespace nkb
