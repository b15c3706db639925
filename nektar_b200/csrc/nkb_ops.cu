// Element operators of the B200 matrix-free path: nkb_op create / apply /
// destroy (the Collections::Operator boundary), geometry packing and the
// shape-generic CUDA kernels. The tuned Hex kernels live in nkb_hex.cu.
//
// Formulation. For every element the reference's fused Helmholtz kernel
// (MatrixFreeOps/Helmholtz.h:549-599) computes
//   y = IP(lambda J w u; B) + sum_a IP(J w (G grad u)_a; B with dB in dir a)
// with u = BwdTrans(x) and G the DiffusionCoeff metric
// (HelmholtzKernels.hpp:390-1114). Because dB = D B (Basis.cpp:493-495), the
// three derivative inner products equal one inner product of
//   f = lambda W u + sum_a D_a^T (G' grad u)_a ,  W = J w0 w1 w2, G' = W G,
// so one BwdTrans, one raw inner product and two collocation derivative
// passes do the work of the reference's one BwdTrans + four inner products.
// W and the six unique entries of G' are packed per quadrature point at
// create time in FP64 (the geometric-factor setup stays FP64).
#include "nkb_internal.h"
#include "nkb_op.h"
#include "nkb_generic_kernel.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace nkb
{

static thread_local std::string g_err;

int SetError(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

void ClearError()
{
    g_err.clear();
}

// ---------------------------------------------------------------------------
// geometry packing (FP64 on the device)
// ---------------------------------------------------------------------------

// Rows a_a of d eta_a / d x_k for the shape at point (i, j, k): the chain rule
// of PhysDerivKernels.hpp:184-344 folded with the derivative factors, the
// same combination HelmholtzKernels.hpp uses for its metric (h0..h3 of
// GetHelmholtz3DHalfSpace, HelmholtzKernels.hpp:1357-1425).
__device__ void ShapeRows(int shape, const double *f, double z0, double z1, double z2, double a[9])
{
    if (shape == NKB_HEX)
    {
        for (int k = 0; k < 3; ++k)
        {
            a[0 + k] = f[k * 3 + 0];
            a[3 + k] = f[k * 3 + 1];
            a[6 + k] = f[k * 3 + 2];
        }
    }
    else if (shape == NKB_TET)
    {
        const double h0 = 0.5 * (1.0 + z0), h1 = 0.5 * (1.0 + z1);
        const double h2 = 2.0 / (1.0 - z1), h3 = 2.0 / (1.0 - z2);
        const double h2h3 = h2 * h3, h1h3 = h1 * h3, h0h2h3 = h0 * h2h3;
        for (int k = 0; k < 3; ++k)
        {
            a[0 + k] = fma(f[k * 3 + 0], h2h3, h0h2h3 * (f[k * 3 + 1] + f[k * 3 + 2]));
            a[3 + k] = fma(f[k * 3 + 2], h1h3, f[k * 3 + 1] * h3);
            a[6 + k] = f[k * 3 + 2];
        }
    }
    else
    {
        const double h0 = 0.5 * (1.0 + z0), h1 = 2.0 / (1.0 - z2);
        for (int k = 0; k < 3; ++k)
        {
            a[0 + k] = h1 * (h0 * f[k * 3 + 2] + f[k * 3 + 0]);
            a[3 + k] = f[k * 3 + 1];
            a[6 + k] = f[k * 3 + 2];
        }
    }
}

struct PackArgs
{
    int shape, optype, deformed, nelmt, nq0, nq1, nq2, nt;
    const double *jac, *df;       // Collections layout
    const double *z0, *z1, *z2;   // points
    const double *w0, *w1, *w2;   // scaled weights
    int diff_mode;                // NKB_DIFF_*
    double K[6];                  // d00 d01 d11 d02 d12 d22
    const double *vel;            // LinearADR: V' = (-1/lambda) V, three fields (or NULL)
    double *geo;                  // packed FP64
    float *geo32;                 // optional FP32 copy
    int ncomp;                    // 7 Helmholtz, 10 LinearADR, 9 PhysDeriv /
                                  // IProductWRTDerivBase, 1 IProduct
    long gstride;                 // element stride of the packed arrays
};

__global__ void k_scale(double *v, size_t n, double s)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
         i += size_t(gridDim.x) * blockDim.x)
        v[i] = s * v[i];
}

__global__ void k_pack(PackArgs a)
{
    const long nt  = a.nt;
    const long tot = long(a.nelmt) * nt;
    for (long g = blockIdx.x * long(blockDim.x) + threadIdx.x; g < tot;
         g += long(gridDim.x) * blockDim.x)
    {
        const long e = g / nt, q = g % nt;
        const int i = int(q % a.nq0), j = int((q / a.nq0) % a.nq1), k = int(q / (long(a.nq0) * a.nq1));
        const long ncol = a.deformed ? tot : long(a.nelmt);
        const long col  = a.deformed ? g : e;
        const double J  = a.jac ? a.jac[col] : 1.0;
        double *out     = a.geo + e * a.gstride + q;
        float *out32    = a.geo32 ? a.geo32 + e * a.gstride + q : nullptr;
        if (a.optype == NKB_IPRODUCT)
        {
            double W = J * a.w0[i] * a.w1[j] * a.w2[k];
            out[0]   = W;
            if (out32)
                out32[0] = float(W);
            continue;
        }
        double f[9];
        for (int d = 0; d < 9; ++d)
            f[d] = a.df[d * ncol + col];
        double A[9];
        ShapeRows(a.shape, f, a.z0[i], a.z1[j], a.z2[k], A);
        if (a.optype == NKB_PHYSDERIV || a.optype == NKB_IPRODUCT_DERIV)
        {
            // IProductWRTDerivBase folds the quadrature weight into the rows
            const double W = a.optype == NKB_IPRODUCT_DERIV ? J * a.w0[i] * a.w1[j] * a.w2[k] : 1.0;
            for (int c = 0; c < 9; ++c)
            {
                const double v = a.optype == NKB_IPRODUCT_DERIV ? W * A[c] : A[c];
                out[c * nt]    = v;
                if (out32)
                    out32[c * nt] = float(v);
            }
            continue;
        }
        // Helmholtz: W and W * A K A^T (six unique entries)
        double K[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        if (a.diff_mode != NKB_DIFF_NONE)
        {
            K[0][0] = a.K[0];
            K[0][1] = K[1][0] = a.K[1];
            K[1][1]           = a.K[2];
            K[0][2] = K[2][0] = a.K[3];
            K[1][2] = K[2][1] = a.K[4];
            K[2][2]           = a.K[5];
            // the reference Tet kernel keeps d11 = 1 under variable diffusion
            // (HelmholtzKernels.hpp:453-460 never loads varD11)
            if (a.shape == NKB_TET && a.diff_mode == NKB_DIFF_VAR)
                K[1][1] = 1.0;
        }
        double t[3][3];
        for (int x = 0; x < 3; ++x)
            for (int l = 0; l < 3; ++l)
                t[x][l] = A[x * 3 + 0] * K[0][l] + A[x * 3 + 1] * K[1][l] + A[x * 3 + 2] * K[2][l];
        double G[3][3];
        for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y)
                G[x][y] = t[x][0] * A[y * 3 + 0] + t[x][1] * A[y * 3 + 1] + t[x][2] * A[y * 3 + 2];
        const double W = J * a.w0[i] * a.w1[j] * a.w2[k];
        const double v[7] = {W,           W * G[0][0], W * G[1][1], W * G[2][2],
                             W * G[0][1], W * G[0][2], W * G[1][2]};
        for (int c = 0; c < 7; ++c)
        {
            out[c * nt] = v[c];
            if (out32)
                out32[c * nt] = float(v[c]);
        }
        if (a.optype == NKB_LINEAR_ADR)
        {
            // advection rows W * sum_m A[x*3+m] V'_m: V'.grad_x u = sum_x row_x d_x
            const long fld = long(a.nelmt) * nt;
            double V[3]    = {0.0, 0.0, 0.0};
            if (a.vel)
                for (int m = 0; m < 3; ++m)
                    V[m] = a.vel[m * fld + g];
            for (int x = 0; x < 3; ++x)
            {
                const double r = W * fma(A[x * 3 + 2], V[2], fma(A[x * 3 + 1], V[1], A[x * 3] * V[0]));
                out[(7 + x) * nt] = r;
                if (out32)
                    out32[(7 + x) * nt] = float(r);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// generic kernels
// ---------------------------------------------------------------------------
static Dims MakeDims(const nkb_op *op);

// Diagonal of the element Helmholtz matrix: for every mode m,
// diag_m = sum_q lambda W phi_m^2 + grad phi_m . G' grad phi_m,
// phi_m = BwdTrans(e_m). One CTA per element.
template <int SHAPE, typename T> __global__ void k_diag(GenArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smem       = reinterpret_cast<T *>(smem_raw);
    const Dims &d = a.d;
    const long e  = blockIdx.x;
    if (e >= a.nelmt)
        return;
    using BW = Bwd<SHAPE>;
    T *x = smem, *u = x + d.nc, *wa = u + d.nt, *wb = wa + d.wsz, *red = wb + d.wsz;
    const T *G = a.geo + e * a.gstride;
    for (int m = 0; m < d.nc; ++m)
    {
        for (int l = threadIdx.x; l < d.nc; l += blockDim.x)
            x[l] = (l == m) ? T(1) : T(0);
        __syncthreads();
        for (int l = threadIdx.x; l < BW::SizeA(d); l += blockDim.x)
            BW::A(d, a.t, x, wa, l);
        __syncthreads();
        for (int l = threadIdx.x; l < BW::SizeB(d); l += blockDim.x)
            BW::B(d, a.t, x, wa, wb, l);
        __syncthreads();
        for (int l = threadIdx.x; l < d.nt; l += blockDim.x)
            BW::C(d, a.t, x, wb, u, l);
        __syncthreads();
        // mass part sum W u^2 and Laplacian part sum grad u . G' grad u
        T accm = 0, accl = 0;
        for (int l = threadIdx.x; l < d.nt; l += blockDim.x)
        {
            T q0, q1, q2;
            Grad(d, a.t, u, l, q0, q1, q2);
            const T W = G[l], G00 = G[d.nt + l], G11 = G[2 * d.nt + l], G22 = G[3 * d.nt + l];
            const T G01 = G[4 * d.nt + l], G02 = G[5 * d.nt + l], G12 = G[6 * d.nt + l];
            T v = q0 * fma(G00, q0, 2 * (G01 * q1 + G02 * q2));
            v   = fma(q1, fma(G11, q1, 2 * G12 * q2), v);
            v   = fma(q2, G22 * q2, v);
            accm += W * u[l] * u[l];
            accl += v;
        }
        T *red2           = red + blockDim.x;
        red[threadIdx.x]  = accm;
        red2[threadIdx.x] = accl;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1)
        {
            if (threadIdx.x < s)
            {
                red[threadIdx.x] += red[threadIdx.x + s];
                red2[threadIdx.x] += red2[threadIdx.x + s];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            if (a.out1)
            {
                a.out0[e * d.nc + m] = red[0];
                a.out1[e * d.nc + m] = red2[0];
            }
            else
            {
                a.out0[e * d.nc + m] = fma(a.lambda, red[0], red2[0]);
            }
        }
        __syncthreads();
    }
}

// Hex element diagonals by sum factorisation. With, per direction d, the
// tables a_d = B_d^2, c_d = dB_d^2 and x_d = dB_d B_d (dB = D B, the basis
// derivative at the points; element p, point i at [p*nq + i]):
//   M_pqr = sum_ijk W a0[p,i] a1[q,j] a2[r,k]
//   L_pqr = sum_ijk G'00 c0 a1 a2 + G'11 a0 c1 a2 + G'22 a0 a1 c2
//                   + 2 (G'01 x0 x1 a2 + G'02 x0 a1 x2 + G'12 a0 x1 x2)
// i.e. seven three-stage contractions of packed geometry fields against
// products of 1-D tables, the same work as seven inner products, instead of
// one full operator application per coefficient.
// tab: [d][kind][nm*nq], kind 0 = a, 1 = c, 2 = x
__global__ void k_hex_diag(int nm, int nq, const double *__restrict__ tab,
                           const double *__restrict__ geo, long gstride, long nelmt, double lambda,
                           double *__restrict__ out0, double *__restrict__ out1)
{
    extern __shared__ __align__(16) double sh[];
    const long e = blockIdx.x;
    if (e >= nelmt)
        return;
    const int nq2 = nq * nq, nq3 = nq2 * nq, nc = nm * nm * nm;
    double *t1   = sh;                 // [p][k][j]  nm*nq*nq
    double *t2   = t1 + nm * nq2;      // [p][q][k]  nm*nm*nq
    double *accM = t2 + nm * nm * nq;  // nc
    double *accL = accM + nc;          // nc
    const double *G = geo + e * gstride;
    for (int m = threadIdx.x; m < nc; m += blockDim.x)
        accM[m] = accL[m] = 0.0;
    // (field, table kind per direction, factor, into L)
    const int field[7]   = {0, 1, 2, 3, 4, 5, 6};
    const int kind[7][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                            {2, 2, 0}, {2, 0, 2}, {0, 2, 2}};
    const double fac[7]  = {1, 1, 1, 1, 2, 2, 2};
    const int tabn       = nm * nq;
    for (int t = 0; t < 7; ++t)
    {
        const double *F  = G + field[t] * nq3;
        const double *a0 = tab + (0 * 3 + kind[t][0]) * tabn;
        const double *a1 = tab + (1 * 3 + kind[t][1]) * tabn;
        const double *a2 = tab + (2 * 3 + kind[t][2]) * tabn;
        __syncthreads();
        for (int l = threadIdx.x; l < nm * nq2; l += blockDim.x)
        {
            const int p = l / nq2, kj = l - p * nq2; // kj = k*nq + j
            double s = 0.0;
            for (int i = 0; i < nq; ++i)
                s = fma(F[kj * nq + i], a0[p * nq + i], s);
            t1[l] = s;
        }
        __syncthreads();
        for (int l = threadIdx.x; l < nm * nm * nq; l += blockDim.x)
        {
            const int pq = l / nq, k = l - pq * nq, p = pq / nm, q = pq - p * nm;
            double s = 0.0;
            for (int j = 0; j < nq; ++j)
                s = fma(t1[(p * nq + k) * nq + j], a1[q * nq + j], s);
            t2[l] = s;
        }
        __syncthreads();
        double *acc = t == 0 ? accM : accL;
        for (int m = threadIdx.x; m < nc; m += blockDim.x)
        {
            const int p = m % nm, q = (m / nm) % nm, r = m / (nm * nm);
            double s = 0.0;
            for (int k = 0; k < nq; ++k)
                s = fma(t2[(p * nm + q) * nq + k], a2[r * nq + k], s);
            acc[m] = fma(fac[t], s, acc[m]);
        }
    }
    __syncthreads();
    for (int m = threadIdx.x; m < nc; m += blockDim.x)
    {
        if (out1)
        {
            out0[e * nc + m] = accM[m];
            out1[e * nc + m] = accL[m];
        }
        else
        {
            out0[e * nc + m] = fma(lambda, accM[m], accL[m]);
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static Dims MakeDims(const nkb_op *op)
{
    Dims d;
    d.nm    = op->nm;
    d.nq0   = op->nq[0];
    d.nq1   = op->nq[1];
    d.nq2   = op->nq[2];
    d.nc    = op->nc;
    d.nt    = op->nt;
    d.npair = op->nm * (op->nm + 1) / 2;
    int M   = std::max(op->nm, op->nq[0]);
    d.wsz   = M * M * M + 2 * op->nq[2] + M * M;
    return d;
}

template <typename T> static Tabs<T> MakeTabs(const nkb_op *op)
{
    Tabs<T> t;
    const T *const *B = reinterpret_cast<const T *const *>(
        std::is_same<T, double>::value ? (const void *)op->dB : (const void *)op->fB);
    const T *const *D = reinterpret_cast<const T *const *>(
        std::is_same<T, double>::value ? (const void *)op->dD : (const void *)op->fD);
    t.B0 = B[0];
    t.B1 = B[1];
    t.B2 = B[2];
    t.D0 = D[0];
    t.D1 = D[1];
    t.D2 = D[2];
    return t;
}

size_t GenericSmemBytes(const nkb_op *op, int elem_bytes)
{
    return size_t(ElemSmem(MakeDims(op))) * elem_bytes;
}

template <int OP, typename T> static int LaunchGenericShape(const nkb_op *op, GenArgs<T> a, cudaStream_t s)
{
    switch (op->shape)
    {
        case NKB_HEX:
            return LaunchGenericT<NKB_HEX, OP, T>(op, a, s);
        case NKB_PRISM:
            return LaunchGenericT<NKB_PRISM, OP, T>(op, a, s);
        default:
            return LaunchGenericT<NKB_TET, OP, T>(op, a, s);
    }
}

extern template int LaunchHelmStatic<double>(const nkb_op *, const GenArgs<double> &, cudaStream_t);
// Prism / Tet column kernels (nkb_col_kernel.cuh, nkb_col_f64.cu, nkb_col_f32.cu)
template <typename T> int LaunchColHelm(const nkb_op *op, const GenArgs<T> &a, cudaStream_t s);
extern template int LaunchColHelm<double>(const nkb_op *, const GenArgs<double> &, cudaStream_t);
extern template int LaunchColHelm<float>(const nkb_op *, const GenArgs<float> &, cudaStream_t);
extern template int LaunchHelmStatic<float>(const nkb_op *, const GenArgs<float> &, cudaStream_t);

static bool StaticSizes()
{
    const char *v = std::getenv("NKB_GENERIC_STATIC");
    return !(v && std::strcmp(v, "0") == 0);
}

static bool ColKernels()
{
    const char *v = std::getenv("NKB_COL");
    return !(v && std::strcmp(v, "0") == 0);
}

template <typename T>
int LaunchGeneric(const nkb_op *op, const T *in, T *o0, T *o1, T *o2, const int *gmap,
                  const double *gsign, cudaStream_t s, const int *skip, const double *lambda)
{
    // IProductWRTDerivBase through the one-input entry points: the three
    // fields lie consecutively in `in`
    const long field = long(op->nelmt) * op->nt;
    return LaunchGeneric3<T>(op, in, in + field, in + 2 * field, o0, o1, o2, gmap, gsign, s, skip,
                             lambda);
}

template <typename T>
int LaunchGeneric3(const nkb_op *op, const T *in, const T *in1, const T *in2, T *o0, T *o1, T *o2,
                   const int *gmap, const double *gsign, cudaStream_t s, const int *skip,
                   const double *lambda)
{
    GenArgs<T> a;
    a.d      = MakeDims(op);
    a.t      = MakeTabs<T>(op);
    a.geo    = std::is_same<T, double>::value ? (const T *)op->geo : (const T *)op->geo32;
    a.lambda = T(lambda ? *lambda : op->lambda);
    a.in     = in;
    a.in1    = in1;
    a.in2    = in2;
    a.out0   = o0;
    a.out1   = o1;
    a.out2   = o2;
    a.gmap   = gmap;
    a.gsign  = gsign;
    a.gstride = op->gstride;
    a.nelmt  = op->nelmt;
    a.epb    = 1;
    a.skip   = skip;
    switch (op->optype)
    {
        case NKB_BWDTRANS:
            return LaunchGenericShape<GK_BWD, T>(op, a, s);
        case NKB_IPRODUCT:
            return LaunchGenericShape<GK_IP, T>(op, a, s);
        case NKB_PHYSDERIV:
            return LaunchGenericShape<GK_PD, T>(op, a, s);
        case NKB_IPRODUCT_DERIV:
            return LaunchGenericShape<GK_IPD, T>(op, a, s);
        case NKB_LINEAR_ADR:
            if (ColKernels() && !gmap)
            {
                const int rc = LaunchColHelm<T>(op, a, s);
                if (rc != kNotCovered)
                    return rc;
            }
            return LaunchGenericShape<GK_ADR, T>(op, a, s);
        default:
        {
            if (ColKernels())
            {
                const int rc = LaunchColHelm<T>(op, a, s);
                if (rc != kNotCovered)
                    return rc;
            }
            if (StaticSizes())
            {
                const int rc = LaunchHelmStatic<T>(op, a, s);
                if (rc != kNotCovered)
                    return rc;
            }
            return LaunchGenericShape<GK_HELM, T>(op, a, s);
        }
    }
}

template int LaunchGeneric3<double>(const nkb_op *, const double *, const double *,
                                    const double *, double *, double *, double *, const int *,
                                    const double *, cudaStream_t, const int *, const double *);
template int LaunchGeneric3<float>(const nkb_op *, const float *, const float *, const float *,
                                   float *, float *, float *, const int *, const double *,
                                   cudaStream_t, const int *, const double *);
template int LaunchGeneric<double>(const nkb_op *, const double *, double *, double *, double *,
                                   const int *, const double *, cudaStream_t, const int *,
                                   const double *);
template int LaunchGeneric<float>(const nkb_op *, const float *, float *, float *, float *,
                                  const int *, const double *, cudaStream_t, const int *,
                                  const double *);

static int Repack(nkb_op *op)
{
    PackArgs a;
    std::memset(&a, 0, sizeof(a));
    a.shape     = op->shape;
    a.optype    = op->optype;
    a.deformed  = op->deformed;
    a.nelmt     = op->nelmt;
    a.nq0       = op->nq[0];
    a.nq1       = op->nq[1];
    a.nq2       = op->nq[2];
    a.nt        = op->nt;
    a.jac       = op->djac;
    a.df        = op->ddf;
    a.z0        = op->dz[0];
    a.z1        = op->dz[1];
    a.z2        = op->dz[2];
    a.w0        = op->dw[0];
    a.w1        = op->dw[1];
    a.w2        = op->dw[2];
    a.diff_mode = op->diff_mode;
    for (int c = 0; c < 6; ++c)
        a.K[c] = op->diff[c];
    a.vel     = op->dvel;
    a.geo     = op->geo;
    a.geo32   = op->geo32;
    a.ncomp   = op->ncomp;
    a.gstride = op->gstride;
    if (op->ncomp == 0)
        return NKB_OK;
    long tot = long(op->nelmt) * op->nt;
    int nb   = int(std::min<long>((tot + 255) / 256, 148L * 16));
    k_pack<<<std::max(nb, 1), 256, 0, op->stream>>>(a);
    NKB_CUDA_TRY(cudaGetLastError());
    NKB_CUDA_TRY(cudaStreamSynchronize(op->stream));
    return NKB_OK;
}

// a device copy of n doubles given in host or device memory (FP64: copied as
// they are; FP32: converted on the host)
template <typename T> static int Upload(T **dst, const double *src, size_t n)
{
    NKB_CUDA_TRY(cudaMalloc(dst, n * sizeof(T)));
    if constexpr (std::is_same_v<T, double>)
    {
        // a copy from device memory does not wait for itself: finish it
        // before the pack (on the operator's own stream) reads it and the
        // caller frees the source
        NKB_CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyDefault));
        NKB_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
    }
    else
    {
        std::vector<T> tmp(n);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = T(src[i]);
        NKB_CUDA_TRY(cudaMemcpy(*dst, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    }
    return NKB_OK;
}

} // namespace nkb

using namespace nkb;

extern "C" const char *nkb_last_error(void)
{
    return g_err.c_str();
}

extern "C" const char *nkb_version(void)
{
    static std::string v;
    if (v.empty())
    {
        int rt = 0;
        cudaRuntimeGetVersion(&rt);
        v = "nektar_b200 0.1 (sm_100a, CUDA runtime " + std::to_string(rt) + ")";
    }
    return v.c_str();
}

extern "C" int nkb_op_create(const nkb_op_desc *desc, nkb_op **out)
{
    ClearError();
    if (!desc || !out)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: NULL argument");
    *out = nullptr;
    const int shape = desc->shape, nm = desc->nm;
    if (shape != NKB_HEX && shape != NKB_PRISM && shape != NKB_TET)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: unsupported shape %d", shape);
    if (desc->optype != NKB_BWDTRANS && desc->optype != NKB_HELMHOLTZ &&
        desc->optype != NKB_IPRODUCT && desc->optype != NKB_IPRODUCT_DERIV &&
        desc->optype != NKB_PHYSDERIV && desc->optype != NKB_LINEAR_ADR)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: unsupported operator %d", desc->optype);
    if (nm < 2 || nm > 16 || desc->nelmt < 0)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: nm=%d nelmt=%d out of range", nm,
                        desc->nelmt);
    for (int d = 0; d < 3; ++d)
        if (desc->nq[d] < 2 || desc->nq[d] > 24)
            return SetError(NKB_ERR_INVALID, "nkb_op_create: nq[%d]=%d out of range", d,
                            desc->nq[d]);
    // MatrixFree preconditions (BwdTransKernels.hpp:537-545)
    const int *nq = desc->nq;
    bool ok = (shape == NKB_HEX && nq[0] == nq[1] && nq[0] == nq[2]) ||
              (shape == NKB_PRISM && nq[0] == nq[1] && nq[0] == nq[2] + 1) ||
              (shape == NKB_TET && nq[0] == nq[1] + 1 && nq[0] == nq[2] + 1);
    if (!ok)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: point counts (%d,%d,%d) not homogeneous "
                        "for shape %d", nq[0], nq[1], nq[2], shape);
    if (desc->precision != NKB_FP64 && desc->precision != NKB_FP32)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: bad precision %d", desc->precision);
    const int opt = desc->optype;
    auto need = [&](const void *p, const char *what) -> int {
        if (!p)
            return SetError(NKB_ERR_INVALID, "nkb_op_create: %s is required for operator %d", what,
                            opt);
        return NKB_OK;
    };
    const bool helm_like = opt == NKB_HELMHOLTZ || opt == NKB_LINEAR_ADR;
    const bool weighted  = opt == NKB_IPRODUCT || helm_like || opt == NKB_IPRODUCT_DERIV;
    const bool derived   = opt == NKB_PHYSDERIV || helm_like || opt == NKB_IPRODUCT_DERIV;
    for (int d = 0; d < 3; ++d)
    {
        if (opt != NKB_PHYSDERIV && need(desc->bdata[d], "bdata"))
            return NKB_ERR_INVALID;
        if (weighted && need(desc->w[d], "w"))
            return NKB_ERR_INVALID;
        if (derived && (need(desc->D[d], "D") || need(desc->z[d], "z")))
            return NKB_ERR_INVALID;
    }
    if (weighted && need(desc->jac, "jac"))
        return NKB_ERR_INVALID;
    if (derived && need(desc->df, "df"))
        return NKB_ERR_INVALID;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return SetError(NKB_ERR_NO_DEVICE, "nkb_op_create: no CUDA device");
    if (desc->device < 0 || desc->device >= ndev)
        return SetError(NKB_ERR_INVALID, "nkb_op_create: device %d of %d", desc->device, ndev);
    NKB_CUDA_TRY(cudaSetDevice(desc->device));

    nkb_op *op    = new nkb_op();
    op->shape     = shape;
    op->optype    = opt;
    op->nm        = nm;
    op->nelmt     = desc->nelmt;
    op->deformed  = desc->deformed ? 1 : 0;
    op->precision = desc->precision;
    op->device    = desc->device;
    for (int d = 0; d < 3; ++d)
    {
        op->nq[d]    = nq[d];
        op->ptype[d] = desc->ptype[d];
    }
    op->nc = NumCoeffs(shape, nm);
    if (opt == NKB_LINEAR_ADR)
    {
        // UpdateFactors runs in the reference constructor with the
        // collection's factors; until set_factors: lambda 1, operator -1
        op->factor_lambda = 1.0;
        op->lambda        = -1.0;
    }
    op->nt = nq[0] * nq[1] * nq[2];
    op->ncomp = (opt == NKB_HELMHOLTZ)                                    ? 7
                : (opt == NKB_LINEAR_ADR)                                 ? 10
                : (opt == NKB_PHYSDERIV || opt == NKB_IPRODUCT_DERIV) ? 9
                : (opt == NKB_IPRODUCT ? 1 : 0);
    // element blocks of the packed geometry start on 32-byte boundaries so a
    // bulk (TMA) copy of one element is legal in FP64 and FP32
    op->gstride = (long(op->ncomp) * op->nt + 3) & ~3L;
    int rc = NKB_OK;
    auto fail = [&](int code) {
        nkb_op_destroy(op);
        return code;
    };
    if (cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&op->ev0) != cudaSuccess || cudaEventCreate(&op->ev1) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_op_create: stream/event creation failed"));
    if (cudaMalloc(&op->d_err, 2 * sizeof(int)) != cudaSuccess ||
        cudaMemset(op->d_err, 0, 2 * sizeof(int)) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_op_create: error word"));

    // 1-D tables
    for (int d = 0; d < 3; ++d)
    {
        const size_t nb = size_t(TableModes(shape, d, nm)) * nq[d];
        std::vector<double> zero(std::max<size_t>(nb, size_t(nq[d]) * nq[d]), 0.0);
        const double *B = desc->bdata[d] ? desc->bdata[d] : zero.data();
        const double *D = desc->D[d] ? desc->D[d] : zero.data();
        if ((rc = Upload(&op->dB[d], B, nb)) || (rc = Upload(&op->fB[d], B, nb)) ||
            (rc = Upload(&op->dD[d], D, size_t(nq[d]) * nq[d])) ||
            (rc = Upload(&op->fD[d], D, size_t(nq[d]) * nq[d])))
            return fail(rc);
        std::vector<double> z(nq[d], 0.0), w(nq[d], 0.0);
        if (desc->z[d])
            std::copy(desc->z[d], desc->z[d] + nq[d], z.begin());
        if (desc->w[d])
            for (int i = 0; i < nq[d]; ++i)
                w[i] = WeightFactor(desc->ptype[d]) * desc->w[d][i];
        if ((rc = Upload(&op->dz[d], z.data(), nq[d])) || (rc = Upload(&op->dw[d], w.data(), nq[d])))
            return fail(rc);
        op->hz[d].assign(z.begin(), z.end());
        op->hw[d].assign(w.begin(), w.end());
        op->hB[d].assign(B, B + nb);
        op->hD[d].assign(D, D + size_t(nq[d]) * nq[d]);
    }
    // raw geometry (kept on the device so factor updates can repack)
    const long ncol = op->deformed ? long(op->nelmt) * op->nt : long(op->nelmt);
    if (desc->jac && op->ncomp && op->nelmt)
        if ((rc = Upload(&op->djac, desc->jac, size_t(ncol))))
            return fail(rc);
    if (desc->df && op->ncomp > 1 && op->nelmt)
        if ((rc = Upload(&op->ddf, desc->df, size_t(9) * ncol)))
            return fail(rc);
    if (op->ncomp && op->nelmt)
    {
        const size_t n = size_t(op->nelmt) * op->gstride;
        if (cudaMalloc(&op->geo, n * sizeof(double)) != cudaSuccess)
            return fail(SetError(NKB_ERR_NOMEM, "nkb_op_create: geometry (%zu doubles)", n));
        if (op->precision == NKB_FP32 && cudaMalloc(&op->geo32, n * sizeof(float)) != cudaSuccess)
            return fail(SetError(NKB_ERR_NOMEM, "nkb_op_create: FP32 geometry"));
        if ((rc = Repack(op)))
            return fail(rc);
    }
    if ((rc = BuildTcTables(op)))
        return fail(rc);
    if ((rc = ChooseKernel(op)))
        return fail(rc);
    *out = op;
    return NKB_OK;
}

extern "C" int nkb_op_set_factors(nkb_op *op, double lambda, int diff_mode, const double *diff)
{
    ClearError();
    if (!op)
        return SetError(NKB_ERR_INVALID, "nkb_op_set_factors: NULL op");
    if (diff_mode < NKB_DIFF_NONE || diff_mode > NKB_DIFF_VAR || (diff_mode && !diff))
        return SetError(NKB_ERR_INVALID, "nkb_op_set_factors: bad diffusion mode %d", diff_mode);
    if (op->optype == NKB_LINEAR_ADR)
    {
        // LinearAdvectionDiffusionReaction_MatrixFree::UpdateFactors
        // (LinearAdvectionDiffusionReaction.cpp:578-590): SetLambda(-lambda);
        // it takes no diffusion tensor
        if (diff_mode != NKB_DIFF_NONE)
            return SetError(NKB_ERR_INVALID,
                            "nkb_op_set_factors: LinearADR takes no diffusion tensor");
        if (!(lambda != 0.0))
            return SetError(NKB_ERR_INVALID, "nkb_op_set_factors: LinearADR needs lambda != 0");
        op->factor_lambda = lambda;
        op->lambda        = -1 * lambda;
        return NKB_OK;
    }
    op->lambda = lambda;
    bool repack = (diff_mode != op->diff_mode);
    if (diff_mode)
        for (int c = 0; c < 6; ++c)
            if (diff[c] != op->diff[c])
            {
                repack     = true;
                op->diff[c] = diff[c];
            }
    op->diff_mode = diff_mode;
    if (!diff_mode)
    {
        const double id[6] = {1, 0, 1, 0, 0, 1};
        for (int c = 0; c < 6; ++c)
            op->diff[c] = id[c];
    }
    if (repack && op->optype == NKB_HELMHOLTZ)
    {
        NKB_CUDA_TRY(cudaSetDevice(op->device));
        return Repack(op);
    }
    return NKB_OK;
}

extern "C" int nkb_op_set_varcoeffs(nkb_op *op, const double *velx, const double *vely,
                                    const double *velz, int flags)
{
    ClearError();
    if (!op || !velx || !vely || !velz)
        return SetError(NKB_ERR_INVALID, "nkb_op_set_varcoeffs: NULL argument");
    if (op->optype != NKB_LINEAR_ADR)
        return SetError(NKB_ERR_INVALID, "nkb_op_set_varcoeffs: operator %d takes no velocities",
                        op->optype);
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    const size_t fld = size_t(op->nelmt) * op->nt;
    if (fld == 0)
        return NKB_OK;
    if (!op->dvel && cudaMalloc(&op->dvel, 3 * fld * sizeof(double)) != cudaSuccess)
        return SetError(NKB_ERR_NOMEM, "nkb_op_set_varcoeffs: velocities (%zu doubles)", 3 * fld);
    const double *src[3] = {velx, vely, velz};
    const cudaMemcpyKind kind =
        (flags & NKB_HOST_PTRS) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    // device arrays may still be written by the caller's streams
    if (!(flags & NKB_HOST_PTRS))
        NKB_CUDA_TRY(cudaDeviceSynchronize());
    for (int d = 0; d < 3; ++d)
        NKB_CUDA_TRY(cudaMemcpyAsync(op->dvel + d * fld, src[d], fld * sizeof(double), kind,
                                     op->stream));
    // LinearAdvectionDiffusionReaction.cpp:662-672: scaled by -1/lambda at
    // the time of the update
    const int nb = int(std::min<size_t>((3 * fld + 255) / 256, 148 * 16));
    if (nb > 0) // an empty collection has nothing to scale
        k_scale<<<nb, 256, 0, op->stream>>>(op->dvel, 3 * fld, -1 / op->factor_lambda);
    NKB_CUDA_TRY(cudaGetLastError());
    return Repack(op);
}

// unit input for column j of every element's matrix
__global__ void k_unit_col(long n, int nc, int j, double *__restrict__ x)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        x[i] = (i % nc == j) ? 1.0 : 0.0;
}

// K[e][i][j] = y[e][i], K rows of `stride` doubles (nc, or the width of a
// column group)
__global__ void k_put_col(long n, int stride, int j, const double *__restrict__ y,
                          double *__restrict__ K)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        K[i * stride + j] = y[i];
}

extern "C" int nkb_op_element_matrices(nkb_op *op, double *K, int flags, void *stream)
{
    ClearError();
    if (!op || !K)
        return SetError(NKB_ERR_INVALID, "nkb_op_element_matrices: NULL argument");
    long nin, nout;
    nkb_op_sizes(op, &nin, &nout);
    if (op->precision != NKB_FP64 || nin != nout || op->nelmt == 0 || nin % op->nelmt)
        return SetError(NKB_ERR_INVALID,
                        "nkb_op_element_matrices: needs an FP64 operator with as many outputs "
                        "as inputs per element");
    const int nc  = int(nin / op->nelmt);
    const long n  = nin;
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    cudaStream_t s   = static_cast<cudaStream_t>(stream);
    const bool host  = (flags & NKB_HOST_PTRS) != 0;
    // host K: built a group of columns at a time in a device buffer of at
    // most 1 GiB, each group copied into the strided host rows by one 2-D copy
    const int width  = host ? int(std::max<long>(1, std::min<long>(nc, (1L << 30) / (n * 8)))) : nc;
    double *x = nullptr, *y = nullptr, *dK = host ? nullptr : K;
    auto release = [&]() {
        cudaFree(x);
        cudaFree(y);
        if (host)
            cudaFree(dK);
    };
    if (cudaMalloc(&x, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&y, n * sizeof(double)) != cudaSuccess ||
        (host && cudaMalloc(&dK, size_t(n) * width * sizeof(double)) != cudaSuccess))
    {
        release();
        return SetError(NKB_ERR_NOMEM, "nkb_op_element_matrices: %ld x %d doubles", n, width);
    }
    const int nb   = int(std::min<long>((n + 255) / 256, 148L * 16));
    cudaError_t ce = cudaSuccess;
    for (int j0 = 0; j0 < nc && ce == cudaSuccess; j0 += width)
    {
        const int w = std::min(width, nc - j0);
        for (int j = j0; j < j0 + w; ++j)
        {
            k_unit_col<<<nb, 256, 0, s>>>(n, nc, j, x);
            int rc = LaunchOp<double>(op, x, y, nullptr, nullptr, nullptr, nullptr, s);
            if (rc)
            {
                cudaStreamSynchronize(s);
                release();
                return rc;
            }
            k_put_col<<<nb, 256, 0, s>>>(n, host ? width : nc, host ? j - j0 : j, y, dK);
        }
        ce = cudaGetLastError();
        if (ce == cudaSuccess && host)
            ce = cudaMemcpy2DAsync(K + j0, size_t(nc) * sizeof(double), dK,
                                   size_t(width) * sizeof(double), size_t(w) * sizeof(double),
                                   size_t(n), cudaMemcpyDeviceToHost, s);
    }
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(s);
    release();
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_op_element_matrices: %s", cudaGetErrorString(ce));
    return CheckOpError(op);
}

extern "C" int nkb_op_sizes(const nkb_op *op, long *in_size, long *out_size)
{
    if (!op)
        return SetError(NKB_ERR_INVALID, "nkb_op_sizes: NULL op");
    const long nc = long(op->nelmt) * op->nc, nt = long(op->nelmt) * op->nt;
    long in = nc, out = nc;
    if (op->optype == NKB_BWDTRANS)
        out = nt;
    else if (op->optype == NKB_IPRODUCT)
        in = nt;
    else if (op->optype == NKB_IPRODUCT_DERIV)
        in = 3 * nt;
    else if (op->optype == NKB_PHYSDERIV)
        in = out = nt;
    else if (op->optype == NKB_DENSE_BLOCK)
        out = nt; // rows per element; nc columns
    if (in_size)
        *in_size = in;
    if (out_size)
        *out_size = out;
    return NKB_OK;
}

namespace nkb
{
int CheckOpError(nkb_op *op)
{
    if (!op || !op->d_err)
        return NKB_OK;
    int word = 0;
    NKB_CUDA_TRY(cudaMemcpy(&word, op->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!word)
        return NKB_OK;
    NKB_CUDA_TRY(cudaMemset(op->d_err, 0, sizeof(int)));
    return SetError(NKB_ERR_TIMEOUT,
                    "operator kernel: a bounded wait for the geometry copy gave up (code %d); the "
                    "outputs of the elements it guarded were not written",
                    word);
}
} // namespace nkb

extern "C" int nkb_op_check_error(nkb_op *op)
{
    ClearError();
    if (!op)
        return SetError(NKB_ERR_INVALID, "nkb_op_check_error: NULL op");
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    return CheckOpError(op);
}

extern "C" int nkb_op_set_wait_limit(nkb_op *op, int polls)
{
    ClearError();
    if (!op)
        return SetError(NKB_ERR_INVALID, "nkb_op_set_wait_limit: NULL op");
    if (polls >= (1 << 24))
        return SetError(NKB_ERR_INVALID, "nkb_op_set_wait_limit: %d polls (at most 2^24 - 1)", polls);
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    const int word = polls < 0 ? 0 : polls + 1;
    NKB_CUDA_TRY(cudaMemcpy(op->d_err + 1, &word, sizeof(int), cudaMemcpyHostToDevice));
    return NKB_OK;
}

static int EnsureScratch(nkb_op *op, size_t bytes)
{
    if (op->scratch_bytes >= bytes)
        return NKB_OK;
    if (op->scratch)
        cudaFree(op->scratch);
    op->scratch       = nullptr;
    op->scratch_bytes = 0;
    if (cudaMalloc(&op->scratch, bytes) != cudaSuccess)
        return SetError(NKB_ERR_NOMEM, "nkb_op_apply: staging buffer of %zu bytes", bytes);
    op->scratch_bytes = bytes;
    return NKB_OK;
}

extern "C" int nkb_op_apply(nkb_op *op, const double *in, double *out0, double *out1,
                            double *out2, int flags, void *stream)
{
    ClearError();
    if (!op || !in || !out0)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply: NULL argument");
    if (op->precision != NKB_FP64)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply: FP32 operator; use nkb_op_apply_f32");
    if (op->optype == NKB_PHYSDERIV && (!out1 || !out2))
        return SetError(NKB_ERR_INVALID, "nkb_op_apply: PhysDeriv needs three outputs");
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream); // NULL: legacy default stream
    long nin, nout;
    nkb_op_sizes(op, &nin, &nout);
    const int nouts = op->optype == NKB_PHYSDERIV ? 3 : 1;
    if (flags & NKB_HOST_PTRS)
    {
        const size_t bytes = size_t(nin + nouts * nout) * sizeof(double);
        int rc             = EnsureScratch(op, bytes);
        if (rc)
            return rc;
        double *din = static_cast<double *>(op->scratch);
        double *dout = din + nin;
        NKB_CUDA_TRY(cudaMemcpyAsync(din, in, nin * sizeof(double), cudaMemcpyHostToDevice, s));
        NKB_CUDA_TRY(cudaEventRecord(op->ev0, s));
        rc = LaunchOp<double>(op, din, dout, nouts > 1 ? dout + nout : nullptr,
                              nouts > 2 ? dout + 2 * nout : nullptr, nullptr, nullptr, s);
        if (rc)
            return rc;
        NKB_CUDA_TRY(cudaEventRecord(op->ev1, s));
        double *outs[3] = {out0, out1, out2};
        for (int o = 0; o < nouts; ++o)
            NKB_CUDA_TRY(cudaMemcpyAsync(outs[o], dout + o * nout, nout * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        return CheckOpError(op);
    }
    NKB_CUDA_TRY(cudaEventRecord(op->ev0, s));
    int rc = LaunchOp<double>(op, in, out0, out1, out2, nullptr, nullptr, s);
    if (rc)
        return rc;
    NKB_CUDA_TRY(cudaEventRecord(op->ev1, s));
    return NKB_OK;
}

extern "C" int nkb_op_apply3(nkb_op *op, const double *in0, const double *in1, const double *in2,
                             double *out, int flags, void *stream)
{
    ClearError();
    if (!op || !in0 || !in1 || !in2 || !out)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply3: NULL argument");
    if (op->optype != NKB_IPRODUCT_DERIV)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply3: operator %d takes one input array",
                        op->optype);
    if (op->precision != NKB_FP64)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply3: needs an FP64 operator");
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    cudaStream_t s    = static_cast<cudaStream_t>(stream); // NULL: legacy default stream
    const long field  = long(op->nelmt) * op->nt;
    const long nout   = long(op->nelmt) * op->nc;
    if (flags & NKB_HOST_PTRS)
    {
        int rc = EnsureScratch(op, size_t(3 * field + nout) * sizeof(double));
        if (rc)
            return rc;
        double *din         = static_cast<double *>(op->scratch);
        double *dout        = din + 3 * field;
        const double *hin[3] = {in0, in1, in2};
        for (int f = 0; f < 3; ++f)
            NKB_CUDA_TRY(cudaMemcpyAsync(din + f * field, hin[f], field * sizeof(double),
                                         cudaMemcpyHostToDevice, s));
        NKB_CUDA_TRY(cudaEventRecord(op->ev0, s));
        rc = LaunchGeneric<double>(op, din, dout, nullptr, nullptr, nullptr, nullptr, s);
        if (rc)
            return rc;
        NKB_CUDA_TRY(cudaEventRecord(op->ev1, s));
        NKB_CUDA_TRY(cudaMemcpyAsync(out, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        return CheckOpError(op);
    }
    NKB_CUDA_TRY(cudaEventRecord(op->ev0, s));
    int rc = LaunchGeneric3<double>(op, in0, in1, in2, out, nullptr, nullptr, nullptr, nullptr, s);
    if (rc)
        return rc;
    NKB_CUDA_TRY(cudaEventRecord(op->ev1, s));
    return NKB_OK;
}

extern "C" int nkb_op_apply_f32(nkb_op *op, const float *in, float *out0, float *out1,
                                float *out2, void *stream)
{
    ClearError();
    if (!op || !in || !out0)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply_f32: NULL argument");
    if (op->precision != NKB_FP32)
        return SetError(NKB_ERR_INVALID, "nkb_op_apply_f32: operator is not FP32");
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream); // NULL: legacy default stream
    NKB_CUDA_TRY(cudaEventRecord(op->ev0, s));
    int rc = LaunchOp<float>(op, in, out0, out1, out2, nullptr, nullptr, s);
    if (rc)
        return rc;
    NKB_CUDA_TRY(cudaEventRecord(op->ev1, s));
    return NKB_OK;
}

extern "C" int nkb_op_last_kernel_ms(const nkb_op *op, float *ms)
{
    if (!op || !ms)
        return SetError(NKB_ERR_INVALID, "nkb_op_last_kernel_ms: NULL argument");
    NKB_CUDA_TRY(cudaEventSynchronize(op->ev1));
    NKB_CUDA_TRY(cudaEventElapsedTime(ms, op->ev0, op->ev1));
    return NKB_OK;
}

namespace nkb
{
static int HexDiag(const nkb_op *op, double *d_out, cudaStream_t s, double *d_stiff)
{
    const int nm = op->nm, nq = op->nq[0];
    const size_t tn = size_t(nm) * nq;
    std::vector<double> tab(9 * tn);
    for (int d = 0; d < 3; ++d)
    {
        const std::vector<double> &B = op->hB[d], &D = op->hD[d]; // D[m*nq + i] = l_m'(z_i)
        for (int p = 0; p < nm; ++p)
            for (int i = 0; i < nq; ++i)
            {
                double db = 0.0;
                for (int m = 0; m < nq; ++m)
                    db += D[size_t(m) * nq + i] * B[size_t(p) * nq + m];
                const double b = B[size_t(p) * nq + i];
                tab[(d * 3 + 0) * tn + p * nq + i] = b * b;
                tab[(d * 3 + 1) * tn + p * nq + i] = db * db;
                tab[(d * 3 + 2) * tn + p * nq + i] = db * b;
            }
    }
    double *dtab = nullptr;
    NKB_CUDA_TRY(cudaMallocAsync((void **)&dtab, tab.size() * sizeof(double), s));
    NKB_CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), tab.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
    const int threads = 256;
    const size_t smem =
        (size_t(nm) * nq * nq + size_t(nm) * nm * nq + 2 * size_t(nm) * nm * nm) * sizeof(double);
    cudaError_t ce = cudaFuncSetAttribute(k_hex_diag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(smem));
    if (ce == cudaSuccess && op->nelmt > 0)
    {
        k_hex_diag<<<op->nelmt, threads, smem, s>>>(nm, nq, dtab, op->geo, op->gstride, op->nelmt,
                                                    op->lambda, d_out, d_stiff);
        ce = cudaGetLastError();
    }
    // the host table must outlive the copy: wait before it goes out of scope
    cudaStreamSynchronize(s);
    cudaFreeAsync(dtab, s);
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "Hex diagonal: %s", cudaGetErrorString(ce));
    return NKB_OK;
}

int HelmholtzDiag(const nkb_op *op, double *d_out, cudaStream_t s, double *d_stiff)
{
    if (op->optype == NKB_DENSE_BLOCK)
        return DenseDiag(op, d_out, s, d_stiff);
    if (op->optype != NKB_HELMHOLTZ)
        return SetError(NKB_ERR_INVALID, "Helmholtz diagonal needs a Helmholtz operator");
    if (op->shape == NKB_HEX && op->nq[0] == op->nq[1] && op->nq[0] == op->nq[2])
        return HexDiag(op, d_out, s, d_stiff);
    GenArgs<double> a;
    a.d      = MakeDims(op);
    a.t      = MakeTabs<double>(op);
    a.geo    = op->geo;
    a.lambda = op->lambda;
    a.in     = nullptr;
    a.out0   = d_out;
    a.out1          = d_stiff;
    a.out2          = nullptr;
    a.gmap          = nullptr;
    a.gsign         = nullptr;
    a.gstride       = op->gstride;
    a.nelmt         = op->nelmt;
    a.epb           = 1;
    a.skip          = nullptr;
    const int threads = 128;
    size_t smem = size_t(a.d.nc + a.d.nt + 2 * a.d.wsz + 2 * threads) * sizeof(double);
    void (*kern)(GenArgs<double>) = op->shape == NKB_HEX     ? k_diag<NKB_HEX, double>
                                    : op->shape == NKB_PRISM ? k_diag<NKB_PRISM, double>
                                                             : k_diag<NKB_TET, double>;
    NKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if (op->nelmt > 0)
        kern<<<op->nelmt, threads, smem, s>>>(a);
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}
} // namespace nkb

extern "C" int nkb_op_helmholtz_diag(nkb_op *op, double *diag, int flags, void *stream)
{
    ClearError();
    if (!op || !diag)
        return SetError(NKB_ERR_INVALID, "nkb_op_helmholtz_diag: NULL argument");
    if (op->precision != NKB_FP64)
        return SetError(NKB_ERR_INVALID, "nkb_op_helmholtz_diag: needs an FP64 operator");
    if (op->optype != NKB_HELMHOLTZ && op->optype != NKB_DENSE_BLOCK)
        return SetError(NKB_ERR_INVALID, "nkb_op_helmholtz_diag: operator %d is not Helmholtz",
                        op->optype);
    NKB_CUDA_TRY(cudaSetDevice(op->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream); // NULL: legacy default stream
    const size_t n = size_t(op->nelmt) * op->nc;
    if (flags & NKB_HOST_PTRS)
    {
        int rc = EnsureScratch(op, n * sizeof(double));
        if (rc)
            return rc;
        double *d = static_cast<double *>(op->scratch);
        if ((rc = HelmholtzDiag(op, d, s)))
            return rc;
        NKB_CUDA_TRY(cudaMemcpyAsync(diag, d, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        return NKB_OK;
    }
    return HelmholtzDiag(op, diag, s);
}

extern "C" void nkb_op_destroy(nkb_op *op)
{
    if (!op)
        return;
    cudaSetDevice(op->device);
    for (int d = 0; d < 3; ++d)
    {
        cudaFree(op->dB[d]);
        cudaFree(op->fB[d]);
        cudaFree(op->dD[d]);
        cudaFree(op->fD[d]);
        cudaFree(op->dz[d]);
        cudaFree(op->dw[d]);
    }
    cudaFree(op->djac);
    cudaFree(op->ddf);
    cudaFree(op->dvel);
    cudaFree(op->geo);
    cudaFree(op->geo32);
    cudaFree(op->scratch);
    cudaFree(op->d_err);
    cudaFree(op->tc_tab);
    FreeKernelData(op);
    if (op->ev0)
        cudaEventDestroy(op->ev0);
    if (op->ev1)
        cudaEventDestroy(op->ev1);
    if (op->stream)
        cudaStreamDestroy(op->stream);
    delete op;
}
