/* Test infrastructure only (the oracle). Plain scalar C restatement of the
 * reference's matrix-free operators, one element at a time; see nkoracle.h
 * for layouts. Each routine cites the reference loop nest it restates. This
 * is the checker for the CUDA path, never the thing measured or shipped. */
#include "nkoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum
{
    TET = 5,
    PRISM = 7,
    HEX = 8
};

int or_ncoeffs(int shape, int nm)
{
    /* ShapeType.hpp:214-225 (tet), 366-374 (prism) */
    if (shape == HEX)
        return nm * nm * nm;
    if (shape == PRISM)
        return nm * nm * (nm + 1) / 2;
    return nm * (nm + 1) * (nm + 2) / 6;
}

/* ------------------------------------------------------------------ */
/* BwdTrans, one element                                               */
/* ------------------------------------------------------------------ */

/* BwdTransKernels.hpp:160-227 */
static void bwd_hex(int nm, const int *nq, const double *const *B, const double *in, double *out,
                    double *w0, double *w1)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    /* contract p: sum_irq[(i*nm + r)*nm + q] */
    for (int i = 0, c = 0; i < nq0; ++i)
        for (int r = 0, cin = 0; r < nm; ++r)
            for (int q = 0; q < nm; ++q, ++c)
            {
                double t = in[cin] * B0[i];
                ++cin;
                for (int p = 1; p < nm; ++p, ++cin)
                    t = fma(in[cin], B0[p * nq0 + i], t);
                w0[c] = t;
            }
    /* contract q: sum_jir[(j*nq0 + i)*nm + r] */
    for (int j = 0, c = 0; j < nq1; ++j)
        for (int i = 0, cirq = 0; i < nq0; ++i)
            for (int r = 0; r < nm; ++r, ++c)
            {
                double t = w0[cirq] * B1[j];
                ++cirq;
                for (int q = 1; q < nm; ++q)
                    t = fma(w0[cirq++], B1[q * nq1 + j], t);
                w1[c] = t;
            }
    /* contract r */
    for (int k = 0, c = 0; k < nq2; ++k)
        for (int j = 0, cjir = 0; j < nq1; ++j)
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double t = w1[cjir] * B2[k];
                ++cjir;
                for (int r = 1; r < nm; ++r)
                    t = fma(w1[cjir++], B2[r * nq2 + k], t);
                out[c] = t;
            }
}

/* BwdTransKernels.hpp:231-330 (correct = true: basis 0 is Modified_A) */
static void bwd_tet(int nm, const int *nq, const double *const *B, const double *in, double *out,
                    double *fpq, double *fp)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        int cpq = 0, cpqr = 0, mode = 0;
        for (int p = 0; p < nm; ++p)
            for (int q = 0; q < nm - p; ++q, ++cpq)
            {
                double prod = in[cpqr] * B2[k + nq2 * mode];
                ++mode;
                ++cpqr;
                for (int r = 1; r < nm - p - q; ++r, ++mode, ++cpqr)
                    prod = fma(in[cpqr], B2[k + nq2 * mode], prod);
                fpq[cpq] = prod;
            }
        for (int j = 0; j < nq1; ++j)
        {
            mode = cpq = 0;
            for (int p = 0; p < nm; ++p)
            {
                double prod = fpq[cpq] * B1[mode * nq1 + j];
                ++cpq;
                for (int q = 1; q < nm - p; ++q, ++cpq)
                    prod = fma(fpq[cpq], B1[(mode + q) * nq1 + j], prod);
                fp[p] = prod;
                mode += nm - p;
            }
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double t = B0[i] * fp[0];
                for (int p = 1; p < nm; ++p)
                    t = fma(B0[p * nq0 + i], fp[p], t);
                /* collapsed top vertex, bottom vertex and singular edge */
                double t1 = B0[i] * B1[nq1 + j];
                t1 = fma(B0[nq0 + i], B1[j], t1);
                t1 = fma(B0[nq0 + i], B1[nq1 + j], t1);
                t1 = t1 * B2[nq2 + k];
                t = fma(t1, in[1], t);
                t1 = B0[nq0 + i] * B1[nq1 + j];
                t1 = t1 * B2[k];
                t = fma(in[nm], t1, t);
                for (int r = 1; r < nm - 1; ++r)
                {
                    t1 = B1[nq1 + j] * B0[nq0 + i];
                    t1 = t1 * B2[(r + 1) * nq2 + k];
                    t = fma(in[nm + r], t1, t);
                }
                out[c] = t;
            }
        }
    }
}

/* BwdTransKernels.hpp:334-403 */
static void bwd_prism(int nm, const int *nq, const double *const *B, const double *in,
                      double *out, double *fpq, double *fp)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        int mpqr = 0, mpq = 0, mpr = 0;
        for (int p = 0; p < nm; ++p)
        {
            for (int q = 0; q < nm; ++q, ++mpq)
            {
                double prod = 0.0;
                for (int r = 0; r < nm - p; ++r, ++mpqr)
                    prod = fma(in[mpqr], B2[(mpr + r) * nq2 + k], prod);
                fpq[mpq] = prod;
            }
            mpr += nm - p;
        }
        for (int j = 0; j < nq1; ++j)
        {
            mpq = 0;
            for (int p = 0; p < nm; ++p)
            {
                double prod = 0.0;
                for (int q = 0; q < nm; ++q, ++mpq)
                    prod = fma(fpq[mpq], B1[q * nq1 + j], prod);
                fp[p] = prod;
            }
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double v = 0.0;
                for (int p = 0; p < nm; ++p)
                    v = fma(fp[p], B0[p * nq0 + i], v);
                double b2 = B2[nq2 + k], b0 = B0[nq0 + i];
                for (int q = 0; q < nm; ++q)
                    v = fma(b2 * B1[q * nq1 + j], b0 * in[q * nm + 1], v);
                out[c] = v;
            }
        }
    }
}

static void bwd_elem(int shape, int nm, const int *nq, const double *const *B, const double *in,
                     double *out, double *w0, double *w1)
{
    if (shape == HEX)
        bwd_hex(nm, nq, B, in, out, w0, w1);
    else if (shape == TET)
        bwd_tet(nm, nq, B, in, out, w0, w1);
    else
        bwd_prism(nm, nq, B, in, out, w0, w1);
}

static size_t wsp_size(int nm, const int *nq)
{
    size_t a = (size_t)(nq[0] > nm ? nq[0] : nm);
    return a * a * a + 64;
}

void or_bwdtrans(int shape, int nm, const int *nq, int nelmt, const double *const *B,
                 const double *in, double *out)
{
    const int nc = or_ncoeffs(shape, nm), nt = nq[0] * nq[1] * nq[2];
    double *w0 = malloc(sizeof(double) * wsp_size(nm, nq));
    double *w1 = malloc(sizeof(double) * wsp_size(nm, nq));
    for (int e = 0; e < nelmt; ++e)
        bwd_elem(shape, nm, nq, B, in + (size_t)e * nc, out + (size_t)e * nt, w0, w1);
    free(w0);
    free(w1);
}

/* ------------------------------------------------------------------ */
/* IProduct, one element, with the ScaleAppend modes of                */
/* IProductKernels.hpp:44-64: mode 0 store, 1 store*scale, 2 add,      */
/* 3 add*scale                                                         */
/* ------------------------------------------------------------------ */

static inline void scale_append(double *store, double v, int scale, int append, double s)
{
    if (scale && append)
        *store = fma(v, s, *store);
    else if (append)
        *store = *store + v;
    else if (scale)
        *store = v * s;
    else
        *store = v;
}

#define JAC(idx) (deformed ? jac[idx] : jac[0])

/* IProductKernels.hpp:271-350 */
static void ip_hex(int nm, const int *nq, const double *const *B, const double *const *w,
                   const double *jac, int deformed, const double *in, double *out, int scale,
                   int append, double s, double *skj, double *sk)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    for (int p = 0; p < nm; ++p)
    {
        int ckji = 0, ckj = 0;
        for (int k = 0; k < nq2; ++k)
            for (int j = 0; j < nq1; ++j, ++ckj)
            {
                double sum = 0.0;
                for (int i = 0; i < nq0; ++i, ++ckji)
                {
                    double prod = in[ckji] * B0[i + nq0 * p] * JAC(nq0 * nq1 * k + nq0 * j + i);
                    sum = fma(prod, w[0][i], sum);
                }
                skj[ckj] = sum;
            }
        for (int q = 0; q < nm; ++q)
        {
            ckj = 0;
            for (int k = 0; k < nq2; ++k)
            {
                double sum = 0.0;
                for (int j = 0; j < nq1; ++j, ++ckj)
                    sum = fma(skj[ckj] * B1[q * nq1 + j], w[1][j], sum);
                sk[k] = sum;
            }
            for (int r = 0; r < nm; ++r)
            {
                double sum = 0.0;
                for (int k = 0; k < nq2; ++k)
                    sum = fma(sk[k] * B2[r * nq2 + k], w[2][k], sum);
                scale_append(&out[r * nm * nm + q * nm + p], sum, scale, append, s);
            }
        }
    }
}

/* IProductKernels.hpp:355-514 */
static void ip_tet(int nm, const int *nq, const double *const *B, const double *const *w,
                   const double *jac, int deformed, const double *in, double *out, int scale,
                   int append, double s, double *skj, double *sk)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    const double *w0 = w[0], *w1 = w[1], *w2 = w[2];
    for (int p = 0, mode = 0, mode2 = 0, cpqr = 0; p < nm; ++p)
    {
        int ckji = 0;
        for (int k = 0, ckj = 0; k < nq2; ++k)
            for (int j = 0; j < nq1; ++j, ++ckj)
            {
                double jv = JAC(nq0 * nq1 * k + nq0 * j);
                double sum = in[ckji] * B0[nq0 * p] * jv * w0[0];
                ++ckji;
                for (int i = 1; i < nq0; ++i, ++ckji)
                {
                    jv = JAC(nq0 * nq1 * k + nq0 * j + i);
                    double t = in[ckji] * B0[i + nq0 * p] * jv;
                    sum = fma(t, w0[i], sum);
                }
                skj[ckj] = sum;
            }
        for (int q = 0; q < nm - p; ++q, ++mode)
        {
            int ckj = 0;
            for (int k = 0; k < nq2; ++k)
            {
                double sum = B1[mode * nq1] * skj[ckj] * w1[0];
                ++ckj;
                for (int j = 1; j < nq1; ++j, ++ckj)
                    sum = fma(B1[mode * nq1 + j] * skj[ckj], w1[j], sum);
                sk[k] = sum;
            }
            for (int r = 0; r < nm - p - q; ++r, ++mode2, ++cpqr)
            {
                double t = sk[0] * B2[mode2 * nq2] * w2[0];
                for (int k = 1; k < nq2; ++k)
                    t = fma(sk[k] * B2[mode2 * nq2 + k], w2[k], t);
                scale_append(&out[cpqr], t, scale, append, s);
            }
        }
    }
    /* singular-vertex corrections (correct = true) */
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        double tq2 = w2[k];
        if (!deformed)
            tq2 = tq2 * jac[0];
        for (int j = 0; j < nq1; ++j)
        {
            double tq1 = tq2 * w1[j];
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double tq = tq1 * w0[i];
                double tin = in[c];
                if (deformed)
                    tq = tq * jac[k * nq0 * nq1 + j * nq0 + i];
                double t = B0[i] * B1[nq1 + j];
                t = fma(B0[nq0 + i], B1[j], t);
                t = fma(B0[nq0 + i], B1[nq1 + j], t);
                t = t * B2[nq2 + k];
                t = t * tin;
                scale_append(&out[1], t * tq, scale, 1, s);
                t = B0[nq0 + i] * B1[nq1 + j] * B2[k] * tin;
                scale_append(&out[nm], t * tq, scale, 1, s);
                for (int r = 1; r < nm - 1; ++r)
                {
                    t = B2[(r + 1) * nq2 + k] * B1[nq1 + j] * B0[nq0 + i] * tin;
                    scale_append(&out[nm + r], t * tq, scale, 1, s);
                }
            }
        }
    }
}

/* IProductKernels.hpp:519-655 */
static void ip_prism(int nm, const int *nq, const double *const *B, const double *const *w,
                     const double *jac, int deformed, const double *in, double *out, int scale,
                     int append, double s, double *skj, double *sk)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    const double *B0 = B[0], *B1 = B[1], *B2 = B[2];
    const double *w0 = w[0], *w1 = w[1], *w2 = w[2];
    int mpr = 0, mpqr = 0;
    for (int p = 0; p < nm; ++p)
    {
        int ckji = 0, ckj = 0;
        for (int k = 0; k < nq2; ++k)
            for (int j = 0; j < nq1; ++j, ++ckj)
            {
                double sum = 0.0;
                for (int i = 0; i < nq0; ++i, ++ckji)
                {
                    double prod = B0[nq0 * p + i] * JAC(nq0 * nq1 * k + nq0 * j + i) * w0[i];
                    sum = fma(prod, in[ckji], sum);
                }
                skj[ckj] = sum;
            }
        for (int q = 0; q < nm; ++q)
        {
            ckj = 0;
            for (int k = 0; k < nq2; ++k)
            {
                double sum = 0.0;
                for (int j = 0; j < nq1; ++j, ++ckj)
                    sum = fma(B1[q * nq1 + j] * w1[j], skj[ckj], sum);
                sk[k] = sum;
            }
            for (int r = 0; r < nm - p; ++r, ++mpqr)
            {
                double sum = 0.0;
                for (int k = 0; k < nq2; ++k)
                    sum = fma(B2[(mpr + r) * nq2 + k] * w2[k], sk[k], sum);
                scale_append(&out[mpqr], sum, scale, append, s);
            }
        }
        mpr += nm - p;
    }
    /* singular-edge correction (correct = true) */
    double corr[32];
    for (int q = 0; q < nm; ++q)
        corr[q] = 0.0;
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        double kw = w2[k];
        if (!deformed)
            kw = kw * jac[0];
        for (int j = 0; j < nq1; ++j)
        {
            double kjw = kw * w1[j];
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double prod = kjw * w0[i] * in[c];
                if (deformed)
                    prod *= jac[k * nq1 * nq0 + j * nq0 + i];
                double b2 = B2[nq2 + k], b0 = B0[nq0 + i];
                for (int q = 0; q < nm; ++q)
                    corr[q] = fma(b2 * B1[q * nq1 + j], b0 * prod, corr[q]);
            }
        }
    }
    for (int q = 0; q < nm; ++q)
        scale_append(&out[nm * q + 1], corr[q], scale, 1, s);
}

static void ip_elem(int shape, int nm, const int *nq, const double *const *B,
                    const double *const *w, const double *jac, int deformed, const double *in,
                    double *out, int scale, int append, double s, double *w0, double *w1)
{
    if (shape == HEX)
        ip_hex(nm, nq, B, w, jac, deformed, in, out, scale, append, s, w0, w1);
    else if (shape == TET)
        ip_tet(nm, nq, B, w, jac, deformed, in, out, scale, append, s, w0, w1);
    else
        ip_prism(nm, nq, B, w, jac, deformed, in, out, scale, append, s, w0, w1);
}

void or_iproduct(int shape, int deformed, int nm, const int *nq, int nelmt,
                 const double *const *B, const double *const *w, const double *jac,
                 const double *in, double *out)
{
    const int nc = or_ncoeffs(shape, nm), nt = nq[0] * nq[1] * nq[2];
    double *w0 = malloc(sizeof(double) * wsp_size(nm, nq));
    double *w1 = malloc(sizeof(double) * wsp_size(nm, nq));
    for (int e = 0; e < nelmt; ++e)
    {
        const double *je = deformed ? jac + (size_t)e * nt : jac + e;
        ip_elem(shape, nm, nq, B, w, je, deformed, in + (size_t)e * nt, out + (size_t)e * nc, 0,
                0, 1.0, w0, w1);
    }
    free(w0);
    free(w1);
}

/* ------------------------------------------------------------------ */
/* PhysDeriv                                                           */
/* ------------------------------------------------------------------ */

/* PhysDerivKernels.hpp:436-507: collocation derivatives in the three
 * tensor directions, D column-major. */
static void deriv_tensor(const int *nq, const double *const *D, const double *in, double *d0,
                         double *d1, double *d2)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    for (int i = 0; i < nq0; ++i)
        for (int j = 0; j < nq1 * nq2; ++j)
        {
            double s = 0.0;
            for (int k = 0; k < nq0; ++k)
                s = fma(D[0][k * nq0 + i], in[j * nq0 + k], s);
            d0[j * nq0 + i] = s;
        }
    for (int b = 0; b < nq2; ++b)
    {
        int st = b * nq0 * nq1;
        for (int i = 0; i < nq0; ++i)
            for (int j = 0; j < nq1; ++j)
            {
                double s = 0.0;
                for (int k = 0; k < nq1; ++k)
                    s = fma(in[st + k * nq0 + i], D[1][k * nq1 + j], s);
                d1[st + j * nq0 + i] = s;
            }
    }
    for (int i = 0; i < nq0 * nq1; ++i)
        for (int j = 0; j < nq2; ++j)
        {
            double s = 0.0;
            for (int k = 0; k < nq2; ++k)
                s = fma(in[k * nq0 * nq1 + i], D[2][k * nq2 + j], s);
            d2[j * nq0 * nq1 + i] = s;
        }
}

/* PhysDerivKernels.hpp:184-344: collapsed-coordinate chain rule (tet,
 * prism) followed by the geometric factors. dfe points at this element's
 * first column in the 9-row array of ncol columns. */
static void deriv_chain(int shape, int deformed, const int *nq, const double *const *Z,
                        const double *df, size_t ncol, size_t col0, double *d0, double *d1,
                        double *d2, double *wsp0, double *wsp1)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    if (shape == TET)
    {
        for (int k = 0, e = 0; k < nq2; ++k)
        {
            double x2 = 2.0 / (1.0 - Z[2][k]);
            for (int j = 0; j < nq1; ++j)
            {
                double x1 = 2.0 / (1.0 - Z[1][j]);
                double x = x1 * x2;
                for (int i = 0; i < nq0; ++i, ++e)
                {
                    double v = x * d0[e];
                    d0[e] = v;
                    wsp0[e] = v;
                }
            }
        }
        for (int k = 0, e = 0; k < nq2; ++k)
        {
            double x2 = 2.0 / (1.0 - Z[2][k]);
            for (int j = 0; j < nq1; ++j)
                for (int i = 0; i < nq0; ++i, ++e)
                {
                    double x0 = 0.5 * (1.0 + Z[0][i]);
                    double o0 = x0 * wsp0[e];
                    wsp0[e] = o0;
                    double v1 = x2 * d1[e];
                    d1[e] = o0 + v1;
                    wsp1[e] = v1;
                }
        }
        for (int k = 0, e = 0; k < nq2; ++k)
            for (int j = 0; j < nq1; ++j)
            {
                double x1 = 0.5 * (1.0 + Z[1][j]);
                for (int i = 0; i < nq0; ++i, ++e)
                {
                    double o = fma(wsp1[e], x1, wsp0[e]);
                    o = o + d2[e];
                    d2[e] = o;
                }
            }
    }
    double f[9];
    if (!deformed)
        for (int d = 0; d < 9; ++d)
            f[d] = df[d * ncol + col0];
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        double x2 = (shape == PRISM) ? 2.0 / (1.0 - Z[2][k]) : 0.0;
        for (int j = 0; j < nq1; ++j)
            for (int i = 0; i < nq0; ++i, ++c)
            {
                double a0 = d0[c], a1 = d1[c], a2 = d2[c];
                if (shape == PRISM)
                {
                    a0 *= x2;
                    double x0 = 0.5 * (1.0 + Z[0][i]);
                    a2 = fma(x0, a0, a2);
                }
                if (deformed)
                    for (int d = 0; d < 9; ++d)
                        f[d] = df[d * ncol + col0 + c];
                double o = a0 * f[0];
                o = fma(a1, f[1], o);
                o = fma(a2, f[2], o);
                d0[c] = o;
                o = a0 * f[3];
                o = fma(a1, f[4], o);
                o = fma(a2, f[5], o);
                d1[c] = o;
                o = a0 * f[6];
                o = fma(a1, f[7], o);
                o = fma(a2, f[8], o);
                d2[c] = o;
            }
    }
}

void or_physderiv(int shape, int deformed, const int *nq, int nelmt, const double *const *D,
                  const double *const *Z, const double *df, const double *in, double *out0,
                  double *out1, double *out2)
{
    const int nt = nq[0] * nq[1] * nq[2];
    const size_t ncol = deformed ? (size_t)nelmt * nt : (size_t)nelmt;
    double *wsp0 = malloc(sizeof(double) * nt);
    double *wsp1 = malloc(sizeof(double) * nt);
    for (int e = 0; e < nelmt; ++e)
    {
        size_t off = (size_t)e * nt;
        deriv_tensor(nq, D, in + off, out0 + off, out1 + off, out2 + off);
        deriv_chain(shape, deformed, nq, Z, df, ncol, deformed ? off : (size_t)e, out0 + off,
                    out1 + off, out2 + off, wsp0, wsp1);
    }
    free(wsp0);
    free(wsp1);
}

/* ------------------------------------------------------------------ */
/* Helmholtz                                                           */
/* ------------------------------------------------------------------ */

/* G = J^T K J with J the 3x3 derivative factors for this shape: returns
 * the six unique metric terms g0..g5 = (00, 11, 22, 01, 02, 12) of the
 * reference's DiffusionCoeff*Kernel (HelmholtzKernels.hpp:390-1114). The
 * hex metric terms use the reference's names metric00..metric22; the tet
 * and prism ones fold in the collapsed-coordinate factors h0..h3. */
static void metric_point(int shape, const double *f, const double *dd, int vardiff_tet_quirk,
                         double h0, double h1, double h2, double h3, double *g)
{
    double a[9]; /* rows: d eta_a / d x_k for a = 0,1,2 as a[a*3 + k] */
    if (shape == HEX)
    {
        for (int k = 0; k < 3; ++k)
        {
            a[0 * 3 + k] = f[k * 3 + 0];
            a[1 * 3 + k] = f[k * 3 + 1];
            a[2 * 3 + k] = f[k * 3 + 2];
        }
    }
    else if (shape == TET)
    {
        /* HelmholtzKernels.hpp:409-423 */
        double h2h3 = h2 * h3, h1h3 = h1 * h3, h0h2h3 = h0 * h2h3;
        a[0] = fma(f[0], h2h3, h0h2h3 * (f[1] + f[2]));
        a[1] = fma(f[3], h2h3, h0h2h3 * (f[4] + f[5]));
        a[2] = fma(f[6], h2h3, h0h2h3 * (f[7] + f[8]));
        a[3] = fma(f[2], h1h3, f[1] * h3);
        a[4] = fma(f[5], h1h3, f[4] * h3);
        a[5] = fma(f[8], h1h3, f[7] * h3);
        a[6] = f[2];
        a[7] = f[5];
        a[8] = f[8];
    }
    else
    {
        /* prism, HelmholtzKernels.hpp:620-622; h0 = (1+z0)/2, h1 = 2/(1-z2) */
        a[0] = h1 * (h0 * f[2] + f[0]);
        a[1] = h1 * (h0 * f[5] + f[3]);
        a[2] = h1 * (h0 * f[8] + f[6]);
        a[3] = f[1];
        a[4] = f[4];
        a[5] = f[7];
        a[6] = f[2];
        a[7] = f[5];
        a[8] = f[8];
    }
    if (!dd)
    {
        /* identity diffusion: g_ab = sum_k a[a][k] a[b][k] */
        double m[3][3];
        for (int x = 0; x < 3; ++x)
            for (int y = x; y < 3; ++y)
            {
                double s = a[x * 3] * a[y * 3];
                s = fma(a[x * 3 + 1], a[y * 3 + 1], s);
                s = fma(a[x * 3 + 2], a[y * 3 + 2], s);
                m[x][y] = s;
            }
        g[0] = m[0][0];
        g[1] = m[1][1];
        g[2] = m[2][2];
        g[3] = m[0][1];
        g[4] = m[0][2];
        g[5] = m[1][2];
        return;
    }
    /* anisotropic: K = [[d00 d01 d02][d01 d11 d12][d02 d12 d22]],
     * dd = (d00 d01 d11 d02 d12 d22). The reference tet kernel never loads
     * varD11 from the per-point array (HelmholtzKernels.hpp:453-460) and so
     * keeps d11 = 1 under variable diffusion; vardiff_tet_quirk restates it. */
    double K[3][3];
    K[0][0] = dd[0];
    K[0][1] = K[1][0] = dd[1];
    K[1][1] = vardiff_tet_quirk ? 1.0 : dd[2];
    K[0][2] = K[2][0] = dd[3];
    K[1][2] = K[2][1] = dd[4];
    K[2][2] = dd[5];
    double t[3][3]; /* t[x][l] = sum_k a[x][k] K[k][l] */
    for (int x = 0; x < 3; ++x)
        for (int l = 0; l < 3; ++l)
        {
            double s = a[x * 3 + 0] * K[0][l];
            s = fma(a[x * 3 + 1], K[1][l], s);
            s = fma(a[x * 3 + 2], K[2][l], s);
            t[x][l] = s;
        }
    double m[3][3];
    for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y)
        {
            double s = t[x][0] * a[y * 3 + 0];
            s = fma(t[x][1], a[y * 3 + 1], s);
            s = fma(t[x][2], a[y * 3 + 2], s);
            m[x][y] = s;
        }
    g[0] = m[0][0];
    g[1] = m[1][1];
    g[2] = m[2][2];
    g[3] = m[0][1];
    g[4] = m[0][2];
    g[5] = m[1][2];
}

/* DiffusionCoeff3DKernel: deriv_a <- sum_b G_ab deriv_b at every point */
static void diffusion_coeff(int shape, int deformed, const int *nq, const double *const *Z,
                            const double *df, size_t ncol, size_t col0, int diff_mode,
                            const double *diff, double *d0, double *d1, double *d2)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    double f[9], g[6];
    const double *dd = (diff_mode == 0) ? NULL : diff;
    int quirk = (shape == TET && diff_mode == 2);
    if (!deformed)
        for (int d = 0; d < 9; ++d)
            f[d] = df[d * ncol + col0];
    for (int k = 0, c = 0; k < nq2; ++k)
        for (int j = 0; j < nq1; ++j)
            for (int i = 0; i < nq0; ++i, ++c)
            {
                if (deformed)
                    for (int d = 0; d < 9; ++d)
                        f[d] = df[d * ncol + col0 + c];
                double h0 = 0.5 * (1.0 + Z[0][i]), h1 = 0.0, h2 = 0.0, h3 = 0.0;
                if (shape == TET)
                {
                    /* GetHelmholtz3DHalfSpace, HelmholtzKernels.hpp:1357-1425 */
                    h1 = 0.5 * (1.0 + Z[1][j]);
                    h2 = 2.0 / (1.0 - Z[1][j]);
                    h3 = 2.0 / (1.0 - Z[2][k]);
                }
                else if (shape == PRISM)
                {
                    h1 = 2.0 / (1.0 - Z[2][k]);
                }
                metric_point(shape, f, dd, quirk, h0, h1, h2, h3, g);
                double a0 = d0[c], a1 = d1[c], a2 = d2[c];
                double o = g[0] * a0;
                o = fma(g[3], a1, o);
                o = fma(g[4], a2, o);
                d0[c] = o;
                o = g[3] * a0;
                o = fma(g[1], a1, o);
                o = fma(g[5], a2, o);
                d1[c] = o;
                o = g[4] * a0;
                o = fma(g[5], a1, o);
                o = fma(g[2], a2, o);
                d2[c] = o;
            }
}

/* fusedKernel3D, Helmholtz.h:549-599 */
static void helm_elem(int shape, int deformed, int nm, const int *nq, const double *const *B,
                      const double *const *dB, const double *const *w, const double *const *D,
                      const double *const *Z, const double *jace, const double *df, size_t ncol,
                      size_t col0, double lambda, int diff_mode, const double *diff,
                      const double *in, double *out, double *bwd, double *d0, double *d1,
                      double *d2, double *w0, double *w1)
{
    bwd_elem(shape, nm, nq, B, in, bwd, w0, w1);
    ip_elem(shape, nm, nq, B, w, jace, deformed, bwd, out, 1, 0, lambda, w0, w1);
    deriv_tensor(nq, D, bwd, d0, d1, d2);
    diffusion_coeff(shape, deformed, nq, Z, df, ncol, col0, diff_mode, diff, d0, d1, d2);
    const double *T0[3] = {dB[0], B[1], B[2]};
    const double *T1[3] = {B[0], dB[1], B[2]};
    const double *T2[3] = {B[0], B[1], dB[2]};
    ip_elem(shape, nm, nq, T0, w, jace, deformed, d0, out, 0, 1, 1.0, w0, w1);
    ip_elem(shape, nm, nq, T1, w, jace, deformed, d1, out, 0, 1, 1.0, w0, w1);
    ip_elem(shape, nm, nq, T2, w, jace, deformed, d2, out, 0, 1, 1.0, w0, w1);
}

void or_helmholtz(int shape, int deformed, int nm, const int *nq, int nelmt,
                  const double *const *B, const double *const *dB, const double *const *w,
                  const double *const *D, const double *const *Z, const double *jac,
                  const double *df, double lambda, int diff_mode, const double *diff,
                  const double *in, double *out)
{
    const int nc = or_ncoeffs(shape, nm), nt = nq[0] * nq[1] * nq[2];
    const size_t ncol = deformed ? (size_t)nelmt * nt : (size_t)nelmt;
    double *buf = malloc(sizeof(double) * (6 * (size_t)nt + 2 * wsp_size(nm, nq)));
    double *bwd = buf, *d0 = buf + nt, *d1 = buf + 2 * nt, *d2 = buf + 3 * nt;
    double *w0 = buf + 4 * nt, *w1 = w0 + wsp_size(nm, nq);
    for (int e = 0; e < nelmt; ++e)
    {
        size_t col0 = deformed ? (size_t)e * nt : (size_t)e;
        const double *je = deformed ? jac + (size_t)e * nt : jac + e;
        helm_elem(shape, deformed, nm, nq, B, dB, w, D, Z, je, df, ncol, col0, lambda, diff_mode,
                  diff, in + (size_t)e * nc, out + (size_t)e * nc, bwd, d0, d1, d2, w0, w1);
    }
    free(buf);
}

/* ------------------------------------------------------------------ */
/* LinearAdvectionDiffusionReaction                                    */
/* ------------------------------------------------------------------ */

/* LinearAdvectionDiffusionReactionKernels.hpp Advection{Hex,Tet,Prism}Kernel
 * (:194-278, :280-382, :384-470): bwd += V' . grad_x u from the collocation
 * derivatives d0..d2, V' per point (vel: three fields, field stride fld) */
static void advection(int shape, int deformed, const int *nq, const double *const *Z,
                      const double *df, size_t ncol, size_t col0, const double *vel, size_t fld,
                      size_t off, const double *d0, const double *d1, const double *d2,
                      double *bwd)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    double f[9];
    if (!deformed)
        for (int d = 0; d < 9; ++d)
            f[d] = df[d * ncol + col0];
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        const double z2f = 2.0 / (1.0 - Z[2][k]); /* tet h3, prism h1 */
        for (int j = 0; j < nq1; ++j)
        {
            const double h1 = 0.5 * (1.0 + Z[1][j]), h2 = 2.0 / (1.0 - Z[1][j]);
            for (int i = 0; i < nq0; ++i, ++c)
            {
                if (deformed)
                    for (int d = 0; d < 9; ++d)
                        f[d] = df[d * ncol + col0 + c];
                const double h0 = 0.5 * (1.0 + Z[0][i]);
                double m0 = d0[c], m1 = d1[c], m2 = d2[c];
                if (shape == TET)
                {
                    const double h2h3 = h2 * z2f, h1h3 = h1 * z2f;
                    m0 = h2h3 * d0[c];
                    m1 = m0 * h0;
                    m2 = m1 + d2[c];
                    m2 = fma(h1h3, d1[c], m2);
                    m1 = fma(z2f, d1[c], m1);
                }
                else if (shape == PRISM)
                {
                    m0 = z2f * d0[c];
                    m2 = h0 * m0 + d2[c];
                }
                const double vx = vel[off + c], vy = vel[fld + off + c],
                             vz = vel[2 * fld + off + c];
                double t = f[0] * m0;
                t = fma(f[1], m1, t);
                t = fma(f[2], m2, t);
                t = t * vx;
                double t2 = f[3] * m0;
                t2 = fma(f[4], m1, t2);
                t2 = fma(f[5], m2, t2);
                t = fma(t2, vy, t);
                t2 = f[6] * m0;
                t2 = fma(f[7], m1, t2);
                t2 = fma(f[8], m2, t2);
                t = fma(t2, vz, t);
                bwd[c] = bwd[c] + t;
            }
        }
    }
}

/* LinearAdvectionDiffusionReaction_MatrixFree (Collections
 * LinearAdvectionDiffusionReaction.cpp:578-723) over the MatrixFree
 * fusedKernel3D (LinearAdvectionDiffusionReaction.h:608-670). lambda and vel
 * are the Collections-level eFactorLambda and eVarCoeffVel{X,Y,Z} (three
 * fields of nelmt*nt values); the operator applies lambda' = -lambda and
 * V' = (-1/lambda) V:
 *   out = lambda' (phi, u + V'.grad u) + (grad phi, grad u). */
void or_linear_adr(int shape, int deformed, int nm, const int *nq, int nelmt,
                   const double *const *B, const double *const *dB, const double *const *w,
                   const double *const *D, const double *const *Z, const double *jac,
                   const double *df, double lambda, const double *vel, const double *in,
                   double *out)
{
    const int nc = or_ncoeffs(shape, nm), nt = nq[0] * nq[1] * nq[2];
    const size_t ncol = deformed ? (size_t)nelmt * nt : (size_t)nelmt;
    const size_t fld  = (size_t)nelmt * nt;
    const double lam  = -1 * lambda, s = -1 / lambda;
    double *vs  = malloc(sizeof(double) * 3 * fld);
    double *buf = malloc(sizeof(double) * (6 * (size_t)nt + 2 * wsp_size(nm, nq)));
    double *bwd = buf, *d0 = buf + nt, *d1 = buf + 2 * nt, *d2 = buf + 3 * nt;
    double *w0 = buf + 4 * nt, *w1 = w0 + wsp_size(nm, nq);
    for (size_t i = 0; i < 3 * fld; ++i)
        vs[i] = s * vel[i];
    const double *T0[3] = {dB[0], B[1], B[2]};
    const double *T1[3] = {B[0], dB[1], B[2]};
    const double *T2[3] = {B[0], B[1], dB[2]};
    for (int e = 0; e < nelmt; ++e)
    {
        const size_t off  = (size_t)e * nt;
        const size_t col0 = deformed ? off : (size_t)e;
        const double *je  = deformed ? jac + off : jac + e;
        double *oe        = out + (size_t)e * nc;
        bwd_elem(shape, nm, nq, B, in + (size_t)e * nc, bwd, w0, w1);
        deriv_tensor(nq, D, bwd, d0, d1, d2);
        advection(shape, deformed, nq, Z, df, ncol, col0, vs, fld, off, d0, d1, d2, bwd);
        ip_elem(shape, nm, nq, B, w, je, deformed, bwd, oe, 1, 0, lam, w0, w1);
        diffusion_coeff(shape, deformed, nq, Z, df, ncol, col0, 0, NULL, d0, d1, d2);
        ip_elem(shape, nm, nq, T0, w, je, deformed, d0, oe, 0, 1, 1.0, w0, w1);
        ip_elem(shape, nm, nq, T1, w, je, deformed, d1, oe, 0, 1, 1.0, w0, w1);
        ip_elem(shape, nm, nq, T2, w, je, deformed, d2, oe, 0, 1, 1.0, w0, w1);
    }
    free(buf);
    free(vs);
}

/* ------------------------------------------------------------------ */
/* IProductWRTDerivBase                                                */
/* ------------------------------------------------------------------ */

/* IProductWRTDerivBaseKernels.hpp (Hex / Prism / Tet kernels): the physical
 * vector field (in0, in1, in2) to reference directions with the derivative
 * factors df (and, for Prism / Tet, the collapsed-coordinate factors). */
static void ipd_transform(int shape, int deformed, const int *nq, const double *const *Z,
                          const double *df, size_t ncol, size_t col0, const double *in0,
                          const double *in1, const double *in2, double *t0, double *t1,
                          double *t2)
{
    const int nq0 = nq[0], nq1 = nq[1], nq2 = nq[2];
    double f[9];
    if (!deformed)
        for (int d = 0; d < 9; ++d)
            f[d] = df[d * ncol + col0];
    for (int k = 0, c = 0; k < nq2; ++k)
    {
        const double z2f = 2.0 / (1.0 - Z[2][k]);
        for (int j = 0; j < nq1; ++j)
        {
            const double f3 = (shape == TET) ? 0.5 * (1.0 + Z[1][j]) : 0.0;
            const double f0 = (shape == TET) ? 2.0 * z2f / (1.0 - Z[1][j]) : 0.0;
            for (int i = 0; i < nq0; ++i, ++c)
            {
                if (deformed)
                    for (int d = 0; d < 9; ++d)
                        f[d] = df[d * ncol + col0 + c];
                const double a = in0[c], b = in1[c], g = in2[c];
                double v0 = f[0] * a + f[3] * b + f[6] * g;
                double v1 = f[1] * a + f[4] * b + f[7] * g;
                double v2 = f[2] * a + f[5] * b + f[8] * g;
                if (shape == PRISM)
                {
                    const double hf1 = 0.5 * (1.0 + Z[0][i]);
                    v0 *= z2f;
                    v0 = fma(hf1 * v2, z2f, v0);
                }
                else if (shape == TET)
                {
                    const double f1 = 0.5 * (1.0 + Z[0][i]);
                    v0 = fma(v1 + v2, f1, v0);
                    v0 *= f0;
                    v1 = fma(v2, f3, v1);
                    v1 *= z2f;
                }
                t0[c] = v0;
                t1[c] = v1;
                t2[c] = v2;
            }
        }
    }
}

/* IProductWRTDerivBase.h fusedKernel3D (:789-825): three inner products,
 * each with the basis derivative dB in one direction. The three input
 * fields are consecutive: field f of element e at in + f*nelmt*nt + e*nt. */
void or_iproduct_deriv(int shape, int deformed, int nm, const int *nq, int nelmt,
                       const double *const *B, const double *const *dB, const double *const *w,
                       const double *const *Z, const double *jac, const double *df,
                       const double *in, double *out)
{
    const int nc = or_ncoeffs(shape, nm), nt = nq[0] * nq[1] * nq[2];
    const size_t ncol = deformed ? (size_t)nelmt * nt : (size_t)nelmt;
    const size_t field = (size_t)nelmt * nt;
    double *buf = malloc(sizeof(double) * (3 * (size_t)nt + 2 * wsp_size(nm, nq)));
    double *t0 = buf, *t1 = buf + nt, *t2 = buf + 2 * nt;
    double *w0 = buf + 3 * nt, *w1 = w0 + wsp_size(nm, nq);
    const double *T0[3] = {dB[0], B[1], B[2]};
    const double *T1[3] = {B[0], dB[1], B[2]};
    const double *T2[3] = {B[0], B[1], dB[2]};
    for (int e = 0; e < nelmt; ++e)
    {
        const size_t off = (size_t)e * nt;
        const size_t col0 = deformed ? off : (size_t)e;
        const double *je = deformed ? jac + off : jac + e;
        ipd_transform(shape, deformed, nq, Z, df, ncol, col0, in + off, in + field + off,
                      in + 2 * field + off, t0, t1, t2);
        double *oe = out + (size_t)e * nc;
        ip_elem(shape, nm, nq, T0, w, je, deformed, t0, oe, 0, 0, 1.0, w0, w1);
        ip_elem(shape, nm, nq, T1, w, je, deformed, t1, oe, 0, 1, 1.0, w0, w1);
        ip_elem(shape, nm, nq, T2, w, je, deformed, t2, oe, 0, 1, 1.0, w0, w1);
    }
    free(buf);
}

/* ------------------------------------------------------------------ */
/* Assembly map and CG                                                 */
/* ------------------------------------------------------------------ */

void or_global_to_local(long nloc, const int *map, const double *sign, const double *glob,
                        double *loc)
{
    for (long i = 0; i < nloc; ++i)
        loc[i] = sign ? sign[i] * glob[map[i]] : glob[map[i]];
}

void or_assemble(long nloc, int nglob, const int *map, const double *sign, const double *loc,
                 double *glob)
{
    memset(glob, 0, sizeof(double) * (size_t)nglob);
    for (long i = 0; i < nloc; ++i)
        glob[map[i]] += sign ? sign[i] * loc[i] : loc[i];
}

static void helm_apply(const or_helm_desc *h, const double *in, double *out)
{
    or_helmholtz(h->shape, h->deformed, h->nm, h->nq, h->nelmt, h->B, h->dB, h->w, h->D, h->Z,
                 h->jac, h->df, h->lambda, 0, NULL, in, out);
}

void or_helmholtz_diag(const or_helm_desc *h, double *out)
{
    const int nc = or_ncoeffs(h->shape, h->nm);
    double *e = calloc((size_t)h->nelmt * nc, sizeof(double));
    double *y = malloc(sizeof(double) * (size_t)h->nelmt * nc);
    for (int m = 0; m < nc; ++m)
    {
        for (int el = 0; el < h->nelmt; ++el)
            e[(size_t)el * nc + m] = 1.0;
        helm_apply(h, e, y);
        for (int el = 0; el < h->nelmt; ++el)
        {
            out[(size_t)el * nc + m] = y[(size_t)el * nc + m];
            e[(size_t)el * nc + m] = 0.0;
        }
    }
    free(e);
    free(y);
}

static double dot(long n, const double *a, const double *b)
{
    double s = 0.0;
    for (long i = 0; i < n; ++i)
        s += a[i] * b[i];
    return s;
}

int or_pcg(const or_helm_desc *h, int nglob, int ndir, const int *map, const double *sign,
           const double *diag_inv, const double *b_glob, double *x_glob, double tol, int maxit,
           double *err_out)
{
    const int nc = or_ncoeffs(h->shape, h->nm);
    const long nloc = (long)h->nelmt * nc;
    const int nn = nglob - ndir;
    double *w = calloc(nglob, sizeof(double)), *s = calloc(nglob, sizeof(double));
    double *p = calloc(nn, sizeof(double)), *r = calloc(nn, sizeof(double));
    double *q = calloc(nn, sizeof(double));
    double *wl = malloc(sizeof(double) * nloc), *sl = malloc(sizeof(double) * nloc);
    memcpy(r, b_glob + ndir, sizeof(double) * nn);
    memset(x_glob, 0, sizeof(double) * nglob);
    double eps = dot(nn, r, r);
    double rhs = dot(nglob, b_glob, b_glob);
    rhs = rhs > 1.0e-6 ? rhs : 1.0; /* NekLinSysIter.cpp:96-117 */
    tol = fmax(tol, 1.0e-16);       /* NekLinSysIter.cpp:57 */
    int it = 0;
    if (eps < tol * tol * rhs)
        goto done;
    for (int i = 0; i < nn; ++i)
        w[ndir + i] = r[i] * diag_inv[i];
    or_global_to_local(nloc, map, sign, w, wl);
    helm_apply(h, wl, sl);
    or_assemble(nloc, nglob, map, sign, sl, s);
    double rho = dot(nn, r, w + ndir), mu = dot(nn, s + ndir, w + ndir);
    double beta = 0.0, alpha = rho / mu;
    it = 1;
    while (1)
    {
        if (it > maxit)
            break;
        for (int i = 0; i < nn; ++i)
        {
            p[i] = beta * p[i] + w[ndir + i];
            q[i] = beta * q[i] + s[ndir + i];
            x_glob[ndir + i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        for (int i = 0; i < nn; ++i)
            w[ndir + i] = r[i] * diag_inv[i];
        or_global_to_local(nloc, map, sign, w, wl);
        helm_apply(h, wl, sl);
        or_assemble(nloc, nglob, map, sign, sl, s);
        double rho_new = dot(nn, r, w + ndir);
        mu = dot(nn, s + ndir, w + ndir);
        eps = dot(nn, r, r);
        it++;
        if (eps < tol * tol * rhs)
            break;
        beta = rho_new / rho;
        alpha = rho_new / (mu - rho_new * beta / alpha);
        rho = rho_new;
    }
done:
    if (err_out)
        *err_out = sqrt(eps / rhs);
    free(w);
    free(s);
    free(p);
    free(r);
    free(q);
    free(wl);
    free(sl);
    return it;
}
