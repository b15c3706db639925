// Test infrastructure only: this file is part of the oracle, never of the
// product. It drives the reference's OWN MatrixFreeOps kernels, compiled in
// place from the reference source tree (passed with -I by oracle/Makefile),
// so that the CPU restatement in oracle/nkoracle.c and the CUDA path can be
// checked against the reference's arithmetic, and so that bench.py can time
// the reference CPU path on the host cores.
//
// One translation unit per shape: the reference kernel headers select their
// shape with the SHAPE_TYPE_* / SHAPE_DIMENSION_3D macros, so the Makefile
// compiles this file three times (hex, prism, tet) with NKREF_SHAPE set to the
// exported name prefix.
//
// What is restated here (everything else is the reference's code):
//  * the per-block driver loops of the 3D operators, i.e. interleave -> kernel
//    -> de-interleave with zero padding of the last block:
//      BwdTrans.h:364-420 (operator3D), IProduct.h:410-491 (operator3D),
//      PhysDeriv.h:478-571 (operator3D), Helmholtz.h:374-464 (operator3D) and
//      the fused body Helmholtz.h:549-599 (fusedKernel3D),
//      IProductWRTDerivBase.h:592-694 (operator3D) and :789-825 (fusedKernel3D),
//      LinearAdvectionDiffusionReaction.h:423-606 (operator3D) and :608-670
//      (fusedKernel3D);
//  * the geometry interleave of CoalescedGeomData.cpp:90-159 (GetJacInterLeave)
//    and :265-342 (GetDerivFactorsInterLeave);
//  * the vec_t broadcast of the 1-D tables, Operator.hpp:529-641 (SetUpBdata,
//    SetUpDBdata, SetUpZW, SetUpD). Radau weight scaling is applied by the
//    caller, which passes already-scaled weights;
//  * the Helmholtz factor plumbing of Operator.hpp (SetLambda,
//    SetConstVarDiffusion, SetVarDiffusion) for one collection;
//  * the LinearADR factor plumbing of the Collections operator
//    (LinearAdvectionDiffusionReaction.cpp:578-723: SetLambda(-lambda), the
//    velocities scaled by -1/lambda and interleaved per block).
// The element range is split into per-thread collections (one std::thread
// each), which mirrors MPI ranks each owning a sub-mesh.

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace Nektar
{
using NekDouble = double;
struct OneD
{
};
// Just enough of Nektar's Array<OneD, T> for the kernel signatures in
// HelmholtzKernels.hpp (indexing, size).
template <class Dim, class T> struct Array
{
    T *m_p         = nullptr;
    std::size_t m_n = 0;
    Array() = default;
    Array(T *p, std::size_t n) : m_p(p), m_n(n)
    {
    }
    T &operator[](std::size_t i) const
    {
        return m_p[i];
    }
    std::size_t size() const
    {
        return m_n;
    }
};
} // namespace Nektar

// worker-thread pinning of the timed CPU baseline (ref_common.cpp)
extern "C" void nkref_pin_thread(int t);

#include <LibUtilities/BasicUtils/NekInline.hpp>
#include <LibUtilities/BasicUtils/ShapeType.hpp>
#include <LibUtilities/SimdLib/tinysimd.hpp>

#include <MatrixFreeOps/BwdTransKernels.hpp>
#include <MatrixFreeOps/HelmholtzKernels.hpp>
#include <MatrixFreeOps/IProductKernels.hpp>
#include <MatrixFreeOps/IProductWRTDerivBaseKernels.hpp>
#include <MatrixFreeOps/LinearAdvectionDiffusionReactionKernels.hpp>
#include <MatrixFreeOps/PhysDerivKernels.hpp>

#ifndef NKREF_SHAPE
#error "NKREF_SHAPE must be defined (hex, prism or tet)"
#endif

#define NKREF_CAT2(a, b) a##b
#define NKREF_CAT(a, b) NKREF_CAT2(a, b)
#define NKREF_FN(name) NKREF_CAT(NKREF_CAT(nkref_, NKREF_SHAPE), name)

using namespace Nektar;
using namespace Nektar::MatrixFree;
using VecV = std::vector<vec_t, tinysimd::allocator<vec_t>>;

#if defined(SHAPE_TYPE_HEX)
static constexpr LibUtilities::ShapeType kShape = LibUtilities::eHexahedron;
#elif defined(SHAPE_TYPE_PRISM)
static constexpr LibUtilities::ShapeType kShape = LibUtilities::ePrism;
#elif defined(SHAPE_TYPE_TET)
static constexpr LibUtilities::ShapeType kShape = LibUtilities::eTetrahedron;
#endif

namespace
{

enum
{
    OP_BWDTRANS  = 0,
    OP_HELMHOLTZ = 1,
    OP_LINEAR_ADR = 2,
    OP_IPRODUCT  = 3,
    OP_IPRODUCT_DERIV = 4,
    OP_PHYSDERIV = 5
};

// number of entries of the 1-D table in direction d for this shape
// (Basis.cpp:466-644: Modified_A nm, Modified_B nm(nm+1)/2,
// Modified_C nm(nm+1)(nm+2)/6 modes per point)
std::size_t TableModes(int d, int nm)
{
    int btype = 0; // 0 = A, 1 = B, 2 = C
#if defined(SHAPE_TYPE_PRISM)
    btype = (d == 2) ? 1 : 0;
#elif defined(SHAPE_TYPE_TET)
    btype = d;
#endif
    if (btype == 0)
    {
        return nm;
    }
    if (btype == 1)
    {
        return nm * (nm + 1) / 2;
    }
    return nm * (nm + 1) * (nm + 2) / 6;
}

int NumCoeffs(int nm)
{
#if defined(SHAPE_TYPE_HEX)
    return nm * nm * nm;
#elif defined(SHAPE_TYPE_PRISM)
    return nm * nm * (nm + 1) / 2;
#else
    return nm * (nm + 1) * (nm + 2) / 6;
#endif
}

void Broadcast(const double *src, std::size_t n, VecV &dst)
{
    dst.resize(n);
    for (std::size_t j = 0; j < n; ++j)
    {
        dst[j] = src[j];
    }
}

struct Chunk
{
    int e0 = 0, ne = 0; // element range of this per-thread collection
    int nBlocks = 0, nPads = 0;
    VecV jac, df; // interleaved geometry
    VecV advVel;  // LinearADR: interleaved velocities [block][point][dir]
};

struct RefOp
{
    int op       = 0;
    bool deformed = false;
    int nm       = 0;
    int nq[3]    = {0, 0, 0};
    int nqTot    = 0;
    int nmTot    = 0;
    int nelmt    = 0;
    int nthreads = 1;

    VecV bdata[3], dbdata[3], w[3], Z[3], D[3];
    VecV h0, h1, h2, h3;
    std::vector<double> z[3];

    double lambda       = 1.0;
    bool isConstVarDiff = false;
    bool isVarDiff      = false;
    std::vector<double> constVarDiff = std::vector<double>(6, 0.0);
    std::vector<double> varD[6];

    std::vector<Chunk> chunks;
};

// CoalescedGeomData::GetJacInterLeave (CoalescedGeomData.cpp:90-159) for the
// element range [e0, e0+ne) of a collection: [block][quadpt] with zero padding.
void InterleaveJac(const RefOp &o, const double *jac, Chunk &c)
{
    const int W = vec_t::width;
    alignas(vec_t::alignment) double tmp[vec_t::width];
    if (o.deformed)
    {
        c.jac.resize(std::size_t(c.nBlocks) * o.nqTot);
        for (int b = 0; b < c.nBlocks; ++b)
        {
            for (int q = 0; q < o.nqTot; ++q)
            {
                for (int j = 0; j < W; ++j)
                {
                    int e  = b * W + j;
                    tmp[j] = (e < c.ne) ? jac[std::size_t(c.e0 + e) * o.nqTot + q] : 0.0;
                }
                c.jac[std::size_t(b) * o.nqTot + q].load(tmp);
            }
        }
    }
    else
    {
        c.jac.resize(c.nBlocks);
        for (int b = 0; b < c.nBlocks; ++b)
        {
            for (int j = 0; j < W; ++j)
            {
                int e  = b * W + j;
                tmp[j] = (e < c.ne) ? jac[c.e0 + e] : 0.0;
            }
            c.jac[b].load(tmp);
        }
    }
}

// CoalescedGeomData::GetDerivFactorsInterLeave (CoalescedGeomData.cpp:265-342).
// Input df is Array<TwoD>(9, npts*nElmt) (deformed) or (9, nElmt) (regular),
// row-major: df[dir * ncol + col].
void InterleaveDF(const RefOp &o, const double *df, Chunk &c)
{
    const int W     = vec_t::width;
    const int n_df  = 9;
    alignas(vec_t::alignment) double tmp[vec_t::width];
    if (o.deformed)
    {
        const std::size_t ncol = std::size_t(o.nelmt) * o.nqTot;
        c.df.resize(std::size_t(c.nBlocks) * n_df * o.nqTot);
        std::size_t cnt = 0;
        for (int b = 0; b < c.nBlocks; ++b)
        {
            for (int q = 0; q < o.nqTot; ++q)
            {
                for (int dir = 0; dir < n_df; ++dir, ++cnt)
                {
                    for (int j = 0; j < W; ++j)
                    {
                        int e  = b * W + j;
                        tmp[j] = (e < c.ne)
                                     ? df[dir * ncol + std::size_t(c.e0 + e) * o.nqTot + q]
                                     : 0.0;
                    }
                    c.df[cnt].load(tmp);
                }
            }
        }
    }
    else
    {
        const std::size_t ncol = o.nelmt;
        c.df.resize(std::size_t(c.nBlocks) * n_df);
        for (int b = 0; b < c.nBlocks; ++b)
        {
            for (int dir = 0; dir < n_df; ++dir)
            {
                for (int j = 0; j < W; ++j)
                {
                    int e  = b * W + j;
                    tmp[j] = (e < c.ne) ? df[dir * ncol + c.e0 + e] : 0.0;
                }
                c.df[b * n_df + dir].load(tmp);
            }
        }
    }
}

template <bool DEFORMED> void ApplyBwdTrans(const RefOp &o, const Chunk &c, const double *in, double *out)
{
    const int nm = o.nm, nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W  = vec_t::width;
    std::size_t wsp0Size = 0, wsp1Size = 0;
    BwdTrans3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), tmpIn(o.nmTot), tmpOut(o.nqTot);
    std::vector<double> loc(std::size_t(std::max(o.nmTot, o.nqTot)) * W, 0.0);
    const double *inptr = in + std::size_t(c.e0) * o.nmTot;
    double *outptr      = out + std::size_t(c.e0) * o.nqTot;
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal = std::min(W, c.ne - b * W);
        std::fill(loc.begin(), loc.end(), 0.0);
        std::copy(inptr, inptr + std::size_t(nreal) * o.nmTot, loc.data());
        load_unalign_interleave(loc.data(), o.nmTot, tmpIn);
        BwdTrans3DKernel<kShape>(nm, nm, nm, nq0, nq1, nq2, true, tmpIn, o.bdata[0], o.bdata[1],
                                 o.bdata[2], wsp0, wsp1, tmpOut);
        deinterleave_unalign_store(tmpOut, o.nqTot, loc.data());
        std::copy(loc.data(), loc.data() + std::size_t(nreal) * o.nqTot, outptr);
        inptr += std::size_t(W) * o.nmTot;
        outptr += std::size_t(W) * o.nqTot;
    }
}

template <bool DEFORMED> void ApplyIProduct(const RefOp &o, const Chunk &c, const double *in, double *out)
{
    const int nm = o.nm, nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W  = vec_t::width;
    std::size_t wsp0Size = 0, wsp1Size = 0, wsp2Size = 0;
    IProduct3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size, wsp2Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), wsp2(std::max<std::size_t>(wsp2Size, nm)), tmpIn(o.nqTot),
        tmpOut(o.nmTot);
    std::vector<double> loc(std::size_t(std::max(o.nmTot, o.nqTot)) * W, 0.0);
    const double *inptr = in + std::size_t(c.e0) * o.nqTot;
    double *outptr      = out + std::size_t(c.e0) * o.nmTot;
    const vec_t *jac_ptr = c.jac.data();
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal = std::min(W, c.ne - b * W);
        std::fill(loc.begin(), loc.end(), 0.0);
        std::copy(inptr, inptr + std::size_t(nreal) * o.nqTot, loc.data());
        load_unalign_interleave(loc.data(), o.nqTot, tmpIn);
        IProduct3DKernel<kShape, false, false, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, tmpIn,
                                                         o.bdata[0], o.bdata[1], o.bdata[2], o.w[0],
                                                         o.w[1], o.w[2], jac_ptr, wsp0, wsp1, wsp2,
                                                         tmpOut);
        deinterleave_unalign_store(tmpOut, o.nmTot, loc.data());
        std::copy(loc.data(), loc.data() + std::size_t(nreal) * o.nmTot, outptr);
        inptr += std::size_t(W) * o.nqTot;
        outptr += std::size_t(W) * o.nmTot;
        jac_ptr += DEFORMED ? o.nqTot : 1;
    }
}

template <bool DEFORMED>
void ApplyPhysDeriv(const RefOp &o, const Chunk &c, const double *in, double *out0, double *out1,
                    double *out2)
{
    const int nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W   = vec_t::width;
    constexpr int ndf = 9;
    std::size_t wsp0Size = 0, wsp1Size = 0;
    PhysDeriv3DWorkspace<kShape>(nq0, nq1, nq2, wsp0Size, wsp1Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), tmpIn(o.nqTot), d0(o.nqTot), d1(o.nqTot), d2(o.nqTot);
    std::vector<double> loc(std::size_t(o.nqTot) * W, 0.0);
    const std::size_t off = std::size_t(c.e0) * o.nqTot;
    const double *inptr   = in + off;
    double *o0 = out0 + off, *o1 = out1 + off, *o2 = out2 + off;
    const vec_t *df_ptr = c.df.data();
    vec_t df_tmp[ndf]   = {};
    const std::size_t dfSize = DEFORMED ? std::size_t(ndf) * o.nqTot : ndf;
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal = std::min(W, c.ne - b * W);
        std::size_t n = std::size_t(nreal) * o.nqTot;
        std::fill(loc.begin(), loc.end(), 0.0);
        std::copy(inptr, inptr + n, loc.data());
        load_unalign_interleave(loc.data(), o.nqTot, tmpIn);
        PhysDerivTensor3DKernel(nq0, nq1, nq2, tmpIn, o.D[0], o.D[1], o.D[2], d0, d1, d2);
        PhysDeriv3DKernel<DEFORMED>(nq0, nq1, nq2, o.Z[0], o.Z[1], o.Z[2], df_ptr, df_tmp, wsp0,
                                    wsp1, d0, d1, d2);
        deinterleave_unalign_store(d0, o.nqTot, loc.data());
        std::copy(loc.data(), loc.data() + n, o0);
        deinterleave_unalign_store(d1, o.nqTot, loc.data());
        std::copy(loc.data(), loc.data() + n, o1);
        deinterleave_unalign_store(d2, o.nqTot, loc.data());
        std::copy(loc.data(), loc.data() + n, o2);
        inptr += std::size_t(W) * o.nqTot;
        o0 += std::size_t(W) * o.nqTot;
        o1 += std::size_t(W) * o.nqTot;
        o2 += std::size_t(W) * o.nqTot;
        df_ptr += dfSize;
    }
}

template <bool DEFORMED> void ApplyHelmholtz(const RefOp &o, const Chunk &c, const double *in, double *out)
{
    const int nm = o.nm, nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W  = vec_t::width;
    constexpr int ndf = 9;
    std::size_t wsp0Size = 0, wsp1Size = 0, wsp2Size = 0;
    BwdTrans3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size);
    IProduct3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size, wsp2Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), wsp2(std::max<std::size_t>(wsp2Size, nm));
    VecV tmpIn(o.nmTot), tmpOut(o.nmTot), bwd(o.nqTot), deriv0(o.nqTot), deriv1(o.nqTot),
        deriv2(o.nqTot);
    std::vector<double> loc(std::size_t(o.nmTot) * W, 0.0);

    // Factor arrays in the form the kernels take (Operator.hpp Helmholtz class)
    Array<OneD, NekDouble> cvd(const_cast<double *>(o.constVarDiff.data()), 6);
    Array<OneD, NekDouble> vd[6];
    for (int i = 0; i < 6; ++i)
    {
        vd[i] = Array<OneD, NekDouble>(const_cast<double *>(o.varD[i].data()), o.varD[i].size());
    }

    const double *inptr  = in + std::size_t(c.e0) * o.nmTot;
    double *outptr       = out + std::size_t(c.e0) * o.nmTot;
    const vec_t *jac_ptr = c.jac.data();
    const vec_t *df_ptr  = c.df.data();
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal = std::min(W, c.ne - b * W);
        std::size_t n = std::size_t(nreal) * o.nmTot;
        std::fill(loc.begin(), loc.end(), 0.0);
        std::copy(inptr, inptr + n, loc.data());
        load_unalign_interleave(loc.data(), o.nmTot, tmpIn);

        // fusedKernel3D (Helmholtz.h:549-599)
        BwdTrans3DKernel<kShape>(nm, nm, nm, nq0, nq1, nq2, true, tmpIn, o.bdata[0], o.bdata[1],
                                 o.bdata[2], wsp0, wsp1, bwd);
        IProduct3DKernel<kShape, true, false, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, bwd,
                                                        o.bdata[0], o.bdata[1], o.bdata[2], o.w[0],
                                                        o.w[1], o.w[2], jac_ptr, wsp0, wsp1, wsp2,
                                                        tmpOut, o.lambda);
        PhysDerivTensor3DKernel(nq0, nq1, nq2, bwd, o.D[0], o.D[1], o.D[2], deriv0, deriv1, deriv2);
        DiffusionCoeff3DKernel<kShape, DEFORMED>(nq0, nq1, nq2, o.isConstVarDiff, cvd, o.isVarDiff,
                                                 vd[0], vd[1], vd[2], vd[3], vd[4], vd[5], df_ptr,
                                                 o.h0, o.h1, o.h2, o.h3, deriv0, deriv1, deriv2);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv0,
                                                        o.dbdata[0], o.bdata[1], o.bdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv1,
                                                        o.bdata[0], o.dbdata[1], o.bdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv2,
                                                        o.bdata[0], o.bdata[1], o.dbdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);

        deinterleave_unalign_store(tmpOut, o.nmTot, loc.data());
        std::copy(loc.data(), loc.data() + n, outptr);
        inptr += std::size_t(W) * o.nmTot;
        outptr += std::size_t(W) * o.nmTot;
        if (DEFORMED)
        {
            jac_ptr += o.nqTot;
            df_ptr += std::size_t(ndf) * o.nqTot;
        }
        else
        {
            ++jac_ptr;
            df_ptr += ndf;
        }
    }
}

// LinearAdvectionDiffusionReaction.h fusedKernel3D (:608-670): BwdTrans, the
// collocation derivatives, bwd += V'.grad u, a lambda'-scaled inner product,
// then the Laplacian terms as in Helmholtz (no diffusion tensor is set by the
// Collections operator).
template <bool DEFORMED> void ApplyLinearADR(const RefOp &o, const Chunk &c, const double *in, double *out)
{
    const int nm = o.nm, nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W  = vec_t::width;
    constexpr int ndf = 9;
    std::size_t wsp0Size = 0, wsp1Size = 0, wsp2Size = 0;
    BwdTrans3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size);
    IProduct3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size, wsp2Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), wsp2(std::max<std::size_t>(wsp2Size, nm));
    VecV tmpIn(o.nmTot), tmpOut(o.nmTot), bwd(o.nqTot), deriv0(o.nqTot), deriv1(o.nqTot),
        deriv2(o.nqTot);
    std::vector<double> loc(std::size_t(o.nmTot) * W, 0.0);
    Array<OneD, NekDouble> cvd(const_cast<double *>(o.constVarDiff.data()), 6);
    Array<OneD, NekDouble> vd[6];
    for (int i = 0; i < 6; ++i)
    {
        vd[i] = Array<OneD, NekDouble>(const_cast<double *>(o.varD[i].data()), o.varD[i].size());
    }
    const double *inptr     = in + std::size_t(c.e0) * o.nmTot;
    double *outptr          = out + std::size_t(c.e0) * o.nmTot;
    const vec_t *jac_ptr    = c.jac.data();
    const vec_t *df_ptr     = c.df.data();
    const vec_t *advVel_ptr = c.advVel.data();
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal     = std::min(W, c.ne - b * W);
        std::size_t n = std::size_t(nreal) * o.nmTot;
        std::fill(loc.begin(), loc.end(), 0.0);
        std::copy(inptr, inptr + n, loc.data());
        load_unalign_interleave(loc.data(), o.nmTot, tmpIn);
        BwdTrans3DKernel<kShape>(nm, nm, nm, nq0, nq1, nq2, true, tmpIn, o.bdata[0], o.bdata[1],
                                 o.bdata[2], wsp0, wsp1, bwd);
        PhysDerivTensor3DKernel(nq0, nq1, nq2, bwd, o.D[0], o.D[1], o.D[2], deriv0, deriv1, deriv2);
        Advection3DKernel<kShape, DEFORMED>(nq0, nq1, nq2, advVel_ptr, df_ptr, o.h0, o.h1, o.h2,
                                            o.h3, deriv0, deriv1, deriv2, bwd);
        IProduct3DKernel<kShape, true, false, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, bwd,
                                                        o.bdata[0], o.bdata[1], o.bdata[2], o.w[0],
                                                        o.w[1], o.w[2], jac_ptr, wsp0, wsp1, wsp2,
                                                        tmpOut, o.lambda);
        DiffusionCoeff3DKernel<kShape, DEFORMED>(nq0, nq1, nq2, o.isConstVarDiff, cvd, o.isVarDiff,
                                                 vd[0], vd[1], vd[2], vd[3], vd[4], vd[5], df_ptr,
                                                 o.h0, o.h1, o.h2, o.h3, deriv0, deriv1, deriv2);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv0,
                                                        o.dbdata[0], o.bdata[1], o.bdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv1,
                                                        o.bdata[0], o.dbdata[1], o.bdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, deriv2,
                                                        o.bdata[0], o.bdata[1], o.dbdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        deinterleave_unalign_store(tmpOut, o.nmTot, loc.data());
        std::copy(loc.data(), loc.data() + n, outptr);
        inptr += std::size_t(W) * o.nmTot;
        outptr += std::size_t(W) * o.nmTot;
        advVel_ptr += std::size_t(3) * o.nqTot;
        if (DEFORMED)
        {
            jac_ptr += o.nqTot;
            df_ptr += std::size_t(ndf) * o.nqTot;
        }
        else
        {
            ++jac_ptr;
            df_ptr += ndf;
        }
    }
}

// IProductWRTDerivBase.h fusedKernel3D (:789-825): the physical vector field
// to reference directions (IProductWRTDerivBase3DKernel, with the collapsed
// factors of Prism/Tet), then three inner products, each with the basis
// derivative in one direction. The three input fields are consecutive in
// `in` (field f of element e at in + f*nelmt*nqTot + e*nqTot).
template <bool DEFORMED>
void ApplyIProductDeriv(const RefOp &o, const Chunk &c, const double *in, double *out)
{
    const int nm = o.nm, nq0 = o.nq[0], nq1 = o.nq[1], nq2 = o.nq[2];
    const int W  = vec_t::width;
    constexpr int ndf = 9;
    std::size_t wsp0Size = 0, wsp1Size = 0, wsp2Size = 0;
    IProduct3DWorkspace<kShape>(nm, nm, nm, nq0, nq1, nq2, wsp0Size, wsp1Size, wsp2Size);
    VecV wsp0(wsp0Size), wsp1(wsp1Size), wsp2(std::max<std::size_t>(wsp2Size, nm));
    VecV tIn0(o.nqTot), tIn1(o.nqTot), tIn2(o.nqTot), t0(o.nqTot), t1(o.nqTot), t2(o.nqTot),
        tmpOut(o.nmTot);
    std::vector<double> loc(std::size_t(std::max(o.nmTot, o.nqTot)) * W, 0.0);
    const std::size_t field = std::size_t(o.nelmt) * o.nqTot;
    const double *inptr     = in + std::size_t(c.e0) * o.nqTot;
    double *outptr          = out + std::size_t(c.e0) * o.nmTot;
    const vec_t *jac_ptr    = c.jac.data();
    const vec_t *df_ptr     = c.df.data();
    VecV *tins[3]           = {&tIn0, &tIn1, &tIn2};
    for (int b = 0; b < c.nBlocks; ++b)
    {
        int nreal = std::min(W, c.ne - b * W);
        for (int f = 0; f < 3; ++f)
        {
            std::fill(loc.begin(), loc.end(), 0.0);
            const double *src = inptr + f * field;
            std::copy(src, src + std::size_t(nreal) * o.nqTot, loc.data());
            load_unalign_interleave(loc.data(), o.nqTot, *tins[f]);
        }
        IProductWRTDerivBase3DKernel<kShape, DEFORMED>(nq0, nq1, nq2, df_ptr, o.Z[0], o.Z[1],
                                                       o.Z[2], tIn0, tIn1, tIn2, t0, t1, t2);
        IProduct3DKernel<kShape, false, false, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, t0,
                                                         o.dbdata[0], o.bdata[1], o.bdata[2],
                                                         o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                         wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, t1,
                                                        o.bdata[0], o.dbdata[1], o.bdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        IProduct3DKernel<kShape, false, true, DEFORMED>(nm, nm, nm, nq0, nq1, nq2, true, t2,
                                                        o.bdata[0], o.bdata[1], o.dbdata[2],
                                                        o.w[0], o.w[1], o.w[2], jac_ptr, wsp0,
                                                        wsp1, wsp2, tmpOut);
        deinterleave_unalign_store(tmpOut, o.nmTot, loc.data());
        std::copy(loc.data(), loc.data() + std::size_t(nreal) * o.nmTot, outptr);
        inptr += std::size_t(W) * o.nqTot;
        outptr += std::size_t(W) * o.nmTot;
        if (DEFORMED)
        {
            jac_ptr += o.nqTot;
            df_ptr += std::size_t(ndf) * o.nqTot;
        }
        else
        {
            ++jac_ptr;
            df_ptr += ndf;
        }
    }
}

void ApplyChunk(const RefOp &o, const Chunk &c, const double *in, double *o0, double *o1, double *o2)
{
    if (c.ne == 0)
    {
        return;
    }
    switch (o.op)
    {
        case OP_BWDTRANS:
            o.deformed ? ApplyBwdTrans<true>(o, c, in, o0) : ApplyBwdTrans<false>(o, c, in, o0);
            break;
        case OP_IPRODUCT:
            o.deformed ? ApplyIProduct<true>(o, c, in, o0) : ApplyIProduct<false>(o, c, in, o0);
            break;
        case OP_PHYSDERIV:
            o.deformed ? ApplyPhysDeriv<true>(o, c, in, o0, o1, o2)
                       : ApplyPhysDeriv<false>(o, c, in, o0, o1, o2);
            break;
        case OP_HELMHOLTZ:
            o.deformed ? ApplyHelmholtz<true>(o, c, in, o0) : ApplyHelmholtz<false>(o, c, in, o0);
            break;
        case OP_IPRODUCT_DERIV:
            o.deformed ? ApplyIProductDeriv<true>(o, c, in, o0)
                       : ApplyIProductDeriv<false>(o, c, in, o0);
            break;
        case OP_LINEAR_ADR:
            o.deformed ? ApplyLinearADR<true>(o, c, in, o0) : ApplyLinearADR<false>(o, c, in, o0);
            break;
    }
}

} // namespace

extern "C"
{

    int NKREF_FN(_simd_width)(void)
    {
        return vec_t::width;
    }

    // Build one operator over nelmt elements split into nthreads per-thread
    // collections. Tables follow Nektar's layouts: bdata/dbdata as
    // Basis::GetBdata/GetDbdata, w already scaled as in Operator.hpp:592-625,
    // z = Basis::GetZ, D column-major as Points::GetD()->GetPtr().
    // jac/df as CoalescedGeomData::GetJac / GetDerivFactors.
    void *NKREF_FN(_create)(int op, int deformed, int nm, const int *nq, int nelmt,
                            const double *const *bdata, const double *const *dbdata,
                            const double *const *w, const double *const *z,
                            const double *const *D, const double *jac, const double *df,
                            int nthreads)
    {
        auto *o     = new RefOp();
        o->op       = op;
        o->deformed = deformed != 0;
        o->nm       = nm;
        for (int d = 0; d < 3; ++d)
        {
            o->nq[d] = nq[d];
        }
        o->nqTot    = nq[0] * nq[1] * nq[2];
        o->nmTot    = NumCoeffs(nm);
        o->nelmt    = nelmt;
        o->nthreads = std::max(1, nthreads);

        for (int d = 0; d < 3; ++d)
        {
            std::size_t nb = TableModes(d, nm) * nq[d];
            if (bdata && bdata[d])
            {
                Broadcast(bdata[d], nb, o->bdata[d]);
            }
            if (dbdata && dbdata[d])
            {
                Broadcast(dbdata[d], nb, o->dbdata[d]);
            }
            if (w && w[d])
            {
                Broadcast(w[d], nq[d], o->w[d]);
            }
            if (z && z[d])
            {
                Broadcast(z[d], nq[d], o->Z[d]);
                o->z[d].assign(z[d], z[d] + nq[d]);
            }
            if (D && D[d])
            {
                Broadcast(D[d], std::size_t(nq[d]) * nq[d], o->D[d]);
            }
        }

#if defined(SHAPE_TYPE_TET) || defined(SHAPE_TYPE_PRISM)
        if (op == OP_HELMHOLTZ)
        {
            Array<OneD, const NekDouble> z0(o->z[0].data(), nq[0]), z1(o->z[1].data(), nq[1]),
                z2(o->z[2].data(), nq[2]);
            GetHelmholtz3DHalfSpace<kShape>(nq[0], nq[1], nq[2], z0, z1, z2, o->h0, o->h1, o->h2,
                                            o->h3);
        }
        if (op == OP_LINEAR_ADR)
        {
            Array<OneD, const NekDouble> z0(o->z[0].data(), nq[0]), z1(o->z[1].data(), nq[1]),
                z2(o->z[2].data(), nq[2]);
            GetLinearAdvectionDiffusionReaction3DHalfSpace<kShape>(nq[0], nq[1], nq[2], z0, z1, z2,
                                                                   o->h0, o->h1, o->h2, o->h3);
        }
#endif
        for (int i = 0; i < 6; ++i)
        {
            o->varD[i].assign(o->nqTot, 0.0);
        }

        // split into per-thread collections; every chunk but the last holds a
        // multiple of the vector width, so only the tail is padded
        const int W       = vec_t::width;
        int nblocksTot    = (nelmt + W - 1) / W;
        int nt            = std::min(o->nthreads, std::max(1, nblocksTot));
        o->chunks.resize(nt);
        int e = 0;
        for (int t = 0; t < nt; ++t)
        {
            int blocks = nblocksTot / nt + (t < nblocksTot % nt ? 1 : 0);
            Chunk &c   = o->chunks[t];
            c.e0       = e;
            c.ne       = std::min(blocks * W, nelmt - e);
            c.nBlocks  = (c.ne + W - 1) / W;
            c.nPads    = c.nBlocks * W - c.ne;
            e += c.ne;
            if (jac)
            {
                InterleaveJac(*o, jac, c);
            }
            if (df)
            {
                InterleaveDF(*o, df, c);
            }
            if (op == OP_LINEAR_ADR)
            {
                c.advVel.assign(std::size_t(c.nBlocks) * o->nqTot * 3, vec_t(0.0));
            }
        }
        return o;
    }

    // Helmholtz factors, as Collections::Helmholtz_MatrixFree::UpdateFactors
    // (Helmholtz.cpp:615-691) hands them to MatrixFree::Helmholtz
    // (SetLambda / SetConstVarDiffusion / SetVarDiffusion, Operator.hpp).
    void NKREF_FN(_set_factors)(void *h, double lambda, int isConstVarDiff, const double *diff,
                                int isVarDiff)
    {
        RefOp *o          = static_cast<RefOp *>(h);
        o->lambda         = lambda;
        o->isConstVarDiff = false;
        o->isVarDiff      = false;
        if (isConstVarDiff)
        {
            o->isConstVarDiff = true;
            for (int i = 0; i < 6; ++i)
            {
                o->constVarDiff[i] = diff[i];
            }
        }
        if (isVarDiff)
        {
            o->isVarDiff      = true;
            o->isConstVarDiff = false;
            for (int i = 0; i < 6; ++i)
            {
                std::fill(o->varD[i].begin(), o->varD[i].end(), diff[i]);
            }
        }
    }

    // LinearAdvectionDiffusionReaction_MatrixFree::UpdateFactors then
    // ::UpdateVarcoeffs (LinearAdvectionDiffusionReaction.cpp:578-723):
    // lambda' = -lambda; the velocities (vel: three fields of nelmt*nqTot
    // values) scaled by -1/lambda and interleaved as [block][point][dir].
    void NKREF_FN(_set_adr)(void *h, double lambda, const double *vel)
    {
        RefOp *o  = static_cast<RefOp *>(h);
        o->lambda = -1 * lambda;
        const double s         = -1 / lambda;
        const std::size_t fld  = std::size_t(o->nelmt) * o->nqTot;
        const int W            = vec_t::width;
        alignas(vec_t::alignment) double tmp[vec_t::width];
        for (Chunk &c : o->chunks)
        {
            c.advVel.resize(std::size_t(c.nBlocks) * o->nqTot * 3);
            std::size_t cnt = 0;
            for (int b = 0; b < c.nBlocks; ++b)
            {
                for (int q = 0; q < o->nqTot; ++q)
                {
                    for (int dir = 0; dir < 3; ++dir, ++cnt)
                    {
                        for (int j = 0; j < W; ++j)
                        {
                            const int e = b * W + j;
                            tmp[j]      = (e < c.ne)
                                              ? s * vel[dir * fld + std::size_t(c.e0 + e) * o->nqTot + q]
                                              : 0.0;
                        }
                        c.advVel[cnt].load(tmp);
                    }
                }
            }
        }
    }

    void NKREF_FN(_apply)(void *h, const double *in, double *out0, double *out1, double *out2)
    {
        RefOp *o = static_cast<RefOp *>(h);
        if (o->chunks.size() == 1)
        {
            ApplyChunk(*o, o->chunks[0], in, out0, out1, out2);
            return;
        }
        std::vector<std::thread> ts;
        ts.reserve(o->chunks.size());
        int ci = 0;
        for (auto &c : o->chunks)
        {
            const int t = ci++;
            ts.emplace_back([o, &c, in, out0, out1, out2, t] {
                nkref_pin_thread(t);
                ApplyChunk(*o, c, in, out0, out1, out2);
            });
        }
        for (auto &t : ts)
        {
            t.join();
        }
    }

    void NKREF_FN(_destroy)(void *h)
    {
        delete static_cast<RefOp *>(h);
    }
}
