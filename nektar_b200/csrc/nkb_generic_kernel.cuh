// The shape-generic element kernel (one template for all shapes, operators
// and precisions; sizes at run time or, through SDims, at compile time).
// Included by nkb_ops.cu and by the compile-time-size instantiation units.
#pragma once

#include "nkb_generic.cuh"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <algorithm>

namespace nkb
{

enum
{
    GK_BWD  = 0,
    GK_HELM = 1,
    GK_ADR  = 2,
    GK_IP   = 3,
    GK_IPD  = 4,
    GK_PD   = 5,
    GK_DIAG = 9
};

// per-element shared memory: x[nc] u[nt] g0 g1 g2 [nt] wa[wsz] wb[wsz]
template <class D> __host__ __device__ constexpr int ElemSmem(const D &d)
{
    return (d.nc + 4 * d.nt + 2 * d.wsz + 1) & ~1;
}

// the kernel's dims object: the runtime Dims, or a compile-time SDims
template <class D> __device__ __forceinline__ D DimsOf(const Dims &) { return D{}; }
template <> __device__ __forceinline__ Dims DimsOf<Dims>(const Dims &d) { return d; }

template <typename T> struct GenArgs
{
    Dims d;
    Tabs<T> t;
    const T *geo;
    T lambda;
    const T *in;
    const T *in1, *in2; // IProductWRTDerivBase: the second and third input fields
    T *out0, *out1, *out2;
    // optional gather of the input from a global vector: in[e*nc+m] = sign * gvec[map]
    const int *gmap;
    const double *gsign;
    long gstride;
    int nelmt, epb;
    const int *skip;
};

#define NKB_STAGE(SIZE, ...)                                                                     \
    for (int idx = threadIdx.x; idx < ne * (SIZE); idx += blockDim.x)                             \
    {                                                                                             \
        const int le = idx / (SIZE);                                                              \
        const int l  = idx - le * (SIZE);                                                         \
        T *sm        = smem + le * es;                                                            \
        T *x = sm, *u = sm + d.nc, *g0 = u + d.nt, *g1 = g0 + d.nt, *g2 = g1 + d.nt;              \
        T *wa = g2 + d.nt, *wb = wa + d.wsz;                                                      \
        (void)x;                                                                                  \
        (void)u;                                                                                  \
        (void)g0;                                                                                 \
        (void)g1;                                                                                 \
        (void)g2;                                                                                 \
        (void)wa;                                                                                 \
        (void)wb;                                                                                 \
        const long e = e0 + le;                                                                   \
        (void)e;                                                                                  \
        __VA_ARGS__                                                                               \
    }                                                                                             \
    __syncthreads();

template <int SHAPE, int OP, typename T, class D = Dims> __global__ void k_generic(GenArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smem       = reinterpret_cast<T *>(smem_raw);
    const D d     = DimsOf<D>(a.d);
    const int es  = ElemSmem(d);
    const long e0 = long(blockIdx.x) * a.epb;
    const int ne  = int(min(long(a.epb), long(a.nelmt) - e0));
    if (ne <= 0 || (a.skip && *a.skip))
        return;
    using BW = Bwd<SHAPE>;
    using IP = Ipr<SHAPE>;

    if (OP == GK_BWD || OP == GK_HELM || OP == GK_ADR || OP == GK_DIAG)
    {
        if (OP != GK_DIAG)
        {
            NKB_STAGE(d.nc, {
                if (a.gmap)
                {
                    const long gi = e * d.nc + l;
                    const T v = a.in[a.gmap[gi]];
                    x[l]      = a.gsign ? T(a.gsign[gi]) * v : v;
                }
                else
                {
                    x[l] = a.in[e * d.nc + l];
                }
            })
        }
    }
    else if (OP != GK_IPD)
    {
        NKB_STAGE(d.nt, { u[l] = a.in[e * d.nt + l]; })
    }

    if (OP == GK_BWD || OP == GK_HELM || OP == GK_ADR)
    {
        NKB_STAGE(BW::SizeA(d), { BW::A(d, a.t, x, wa, l); })
        NKB_STAGE(BW::SizeB(d), { BW::B(d, a.t, x, wa, wb, l); })
        NKB_STAGE(d.nt, { BW::C(d, a.t, x, wb, u, l); })
        if (OP == GK_BWD)
        {
            NKB_STAGE(d.nt, { a.out0[e * d.nt + l] = u[l]; })
            return;
        }
    }

    if (OP == GK_PD)
    {
        NKB_STAGE(d.nt, {
            T q0, q1, q2;
            Grad(d, a.t, u, l, q0, q1, q2);
            const T *A = a.geo + e * a.gstride + l;
            const long o = e * d.nt + l;
            a.out0[o] = fma(A[6 * d.nt], q2, fma(A[3 * d.nt], q1, A[0] * q0));
            a.out1[o] = fma(A[7 * d.nt], q2, fma(A[4 * d.nt], q1, A[1 * d.nt] * q0));
            a.out2[o] = fma(A[8 * d.nt], q2, fma(A[5 * d.nt], q1, A[2 * d.nt] * q0));
        })
        return;
    }

    if (OP == GK_IP)
    {
        // f = W * in
        NKB_STAGE(d.nt, { u[l] = u[l] * a.geo[e * a.gstride + l]; })
    }

    if (OP == GK_HELM)
    {
        // v = G' grad u, f = lambda W u
        NKB_STAGE(d.nt, {
            T q0, q1, q2;
            Grad(d, a.t, u, l, q0, q1, q2);
            const T *G = a.geo + e * a.gstride + l;
            const T W = G[0], G00 = G[d.nt], G11 = G[2 * d.nt], G22 = G[3 * d.nt];
            const T G01 = G[4 * d.nt], G02 = G[5 * d.nt], G12 = G[6 * d.nt];
            g0[l] = fma(G02, q2, fma(G01, q1, G00 * q0));
            g1[l] = fma(G12, q2, fma(G11, q1, G01 * q0));
            g2[l] = fma(G22, q2, fma(G12, q1, G02 * q0));
            wa[l] = a.lambda * W * u[l];
        })
        NKB_STAGE(d.nt, { u[l] = wa[l] + GradT(d, a.t, g0, g1, g2, l); })
    }

    if (OP == GK_ADR)
    {
        // LinearADR (LinearAdvectionDiffusionReaction.h:608-670): as Helmholtz
        // with lambda' (u + V'.grad u) for the mass term; the packed rows
        // 7..9 carry W A V'
        NKB_STAGE(d.nt, {
            T q0, q1, q2;
            Grad(d, a.t, u, l, q0, q1, q2);
            const T *G = a.geo + e * a.gstride + l;
            const T W = G[0], G00 = G[d.nt], G11 = G[2 * d.nt], G22 = G[3 * d.nt];
            const T G01 = G[4 * d.nt], G02 = G[5 * d.nt], G12 = G[6 * d.nt];
            const T adv = fma(G[9 * d.nt], q2, fma(G[8 * d.nt], q1, G[7 * d.nt] * q0));
            g0[l] = fma(G02, q2, fma(G01, q1, G00 * q0));
            g1[l] = fma(G12, q2, fma(G11, q1, G01 * q0));
            g2[l] = fma(G22, q2, fma(G12, q1, G02 * q0));
            wa[l] = a.lambda * fma(W, u[l], adv);
        })
        NKB_STAGE(d.nt, { u[l] = wa[l] + GradT(d, a.t, g0, g1, g2, l); })
    }

    if (OP == GK_IPD)
    {
        // v_x = sum_m W A[x*3+m] f_m (the packed rows already carry W), then
        // sum_x D_x^T v_x; dB_x = D_x B_x turns the three inner products of
        // IProductWRTDerivBase.h:789-825 into one with B.
        NKB_STAGE(d.nt, {
            const long o = e * d.nt + l;
            const T f0 = a.in[o], f1 = a.in1[o], f2 = a.in2[o];
            const T *P = a.geo + e * a.gstride + l;
            g0[l] = fma(P[2 * d.nt], f2, fma(P[1 * d.nt], f1, P[0] * f0));
            g1[l] = fma(P[5 * d.nt], f2, fma(P[4 * d.nt], f1, P[3 * d.nt] * f0));
            g2[l] = fma(P[8 * d.nt], f2, fma(P[7 * d.nt], f1, P[6 * d.nt] * f0));
        })
        NKB_STAGE(d.nt, { u[l] = GradT(d, a.t, g0, g1, g2, l); })
    }

    if (OP == GK_HELM || OP == GK_ADR || OP == GK_IP || OP == GK_IPD)
    {
        NKB_STAGE(IP::SizeA(d), { IprStageA(d, a.t, u, wa, l); })
        NKB_STAGE(IP::SizeB(d), { IP::B(d, a.t, wa, wb, l); })
        NKB_STAGE(d.nc, { a.out0[e * d.nc + l] = IP::C(d, a.t, wb, l); })
    }
}



// Launch of k_generic for one operator: elements per CTA and threads per CTA
// from the operator's autotuned launch shape (or the defaults).
template <int SHAPE, int OP, typename T, class D = Dims>
int LaunchGenericT(const nkb_op *op, GenArgs<T> a, cudaStream_t s)
{
    const int es      = ElemSmem(a.d);
    const size_t ebyt = size_t(es) * sizeof(T);
    int epb           = int(std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / ebyt)));
    if (op->gen_epb > 0)
        epb = op->gen_epb; // autotuned (checked against the shared-memory limit)
    const int threads = op->gen_threads > 0 ? op->gen_threads : 128;
    a.epb             = epb;
    const size_t smem = ebyt * epb;
    auto kern         = k_generic<SHAPE, OP, T, D>;
    // raise the dynamic shared-memory limit once per instantiation, before any
    // stream capture can contain this launch
    static size_t s_smem_set = 48 * 1024;
    if (smem > s_smem_set)
    {
        NKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        s_smem_set = smem;
    }
    const long nb = (long(a.nelmt) + epb - 1) / epb;
    if (nb > 0)
        kern<<<unsigned(nb), threads, smem, s>>>(a);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

// Prism / Tet Helmholtz with compile-time sizes for the standard point sets
// and nm = 2..11 (instantiated in nkb_gen_f64.cu / nkb_gen_f32.cu). Returns
// kNotCovered, with no error set, for anything else.
constexpr int kNotCovered = 1;

template <int SHAPE, typename T> int LaunchHelmStaticShape(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s)
{
    switch (op->nm)
    {
#define NKB_HS(N)                                                                                  \
    case N: return LaunchGenericT<SHAPE, GK_HELM, T, SDims<SHAPE, N>>(op, a, s);
        NKB_HS(2) NKB_HS(3) NKB_HS(4) NKB_HS(5) NKB_HS(6) NKB_HS(7) NKB_HS(8) NKB_HS(9)
        NKB_HS(10) NKB_HS(11)
#undef NKB_HS
        default: return kNotCovered;
    }
}

template <typename T> int LaunchHelmStatic(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s)
{
    const int nm = op->nm;
    if (op->nq[0] != nm + 1)
        return kNotCovered;
    if (op->shape == NKB_PRISM && op->nq[1] == nm + 1 && op->nq[2] == nm)
        return LaunchHelmStaticShape<NKB_PRISM, T>(op, a, s);
    if (op->shape == NKB_TET && op->nq[1] == nm && op->nq[2] == nm)
        return LaunchHelmStaticShape<NKB_TET, T>(op, a, s);
    return kNotCovered;
}

} // namespace nkb
