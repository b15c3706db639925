/* Test infrastructure only (the oracle): a plain, scalar C restatement of the
 * reference's matrix-free element operators, assembly map and conjugate
 * gradient for Hex / Prism / Tet. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg call it; the product never links it.
 *
 * Layouts follow the reference's Collections interface:
 *  - per-element arrays are contiguous and element-major: in[e*ncoef + m],
 *    phys[e*nqtot + q] with q = (k*nq1 + j)*nq0 + i (i fastest);
 *  - jac: nelmt*nqtot (deformed) or nelmt (regular), CoalescedGeomData::GetJac;
 *  - df:  9 rows of ncol = nelmt*nqtot (deformed) or nelmt (regular), row
 *         dir = k*3 + j holds d xi_j / d x_k, CoalescedGeomData::GetDerivFactors;
 *  - B[d], dB[d]: Basis::GetBdata/GetDbdata (mode-major, point fastest);
 *  - w[d]: weights already multiplied by the Radau factor of SetUpZW;
 *  - D[d]: column-major collocation derivative, D[k*nq + i] = d l_k/dz (z_i).
 * Shapes are numbered as LibUtilities::ShapeType (5 tet, 7 prism, 8 hex).
 */
#ifndef NKORACLE_H
#define NKORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

int or_ncoeffs(int shape, int nm);

void or_bwdtrans(int shape, int nm, const int *nq, int nelmt, const double *const *B,
                 const double *in, double *out);

void or_iproduct(int shape, int deformed, int nm, const int *nq, int nelmt,
                 const double *const *B, const double *const *w, const double *jac,
                 const double *in, double *out);

void or_physderiv(int shape, int deformed, const int *nq, int nelmt, const double *const *D,
                  const double *const *Z, const double *df, const double *in, double *out0,
                  double *out1, double *out2);

/* diff: NULL, or 6 coefficients (d00 d01 d11 d02 d12 d22);
 * diff_mode 0 = identity, 1 = constant anisotropic (SetConstVarDiffusion),
 * 2 = per-point variable diffusion filled with the same 6 values
 * (SetVarDiffusion as Collections::Helmholtz_MatrixFree drives it). */
/* LinearAdvectionDiffusionReaction (LinearAdvectionDiffusionReaction.cpp:578-723,
 * LinearAdvectionDiffusionReaction.h:608-670): lambda and vel (three fields of
 * nelmt*nt values) as the Collections operator receives them */
void or_linear_adr(int shape, int deformed, int nm, const int *nq, int nelmt,
                   const double *const *B, const double *const *dB, const double *const *w,
                   const double *const *D, const double *const *Z, const double *jac,
                   const double *df, double lambda, const double *vel, const double *in,
                   double *out);
/* IProductWRTDerivBase (IProductWRTDerivBase.h:592-825): in holds the three
 * physical fields consecutively (field f of element e at in + f*nelmt*nt + e*nt) */
void or_iproduct_deriv(int shape, int deformed, int nm, const int *nq, int nelmt,
                       const double *const *B, const double *const *dB, const double *const *w,
                       const double *const *Z, const double *jac, const double *df,
                       const double *in, double *out);
void or_helmholtz(int shape, int deformed, int nm, const int *nq, int nelmt,
                  const double *const *B, const double *const *dB, const double *const *w,
                  const double *const *D, const double *const *Z, const double *jac,
                  const double *df, double lambda, int diff_mode, const double *diff,
                  const double *in, double *out);

/* AssemblyMapCG::GlobalToLocal / Assemble (AssemblyMapCG.cpp:2804-2886) */
void or_global_to_local(long nloc, const int *map, const double *sign, const double *glob,
                        double *loc);
void or_assemble(long nloc, int nglob, const int *map, const double *sign, const double *loc,
                 double *glob);

/* NekLinSysIterCG::DoConjugateGradient (NekLinSysIterCG.cpp:118-372) on the
 * global system A = Assemble o blockdiag(H_e) o GlobalToLocal with the
 * Helmholtz element operator of or_helmholtz, Jacobi preconditioner diag_inv
 * (length nglob-ndir). Returns iterations; x_glob gets the solution on
 * [ndir, nglob) and 0 on the Dirichlet part. */
typedef struct
{
    int shape, deformed, nm, nq[3], nelmt;
    const double *B[3], *dB[3], *w[3], *D[3], *Z[3];
    const double *jac, *df;
    double lambda;
} or_helm_desc;

int or_pcg(const or_helm_desc *h, int nglob, int ndir, const int *map, const double *sign,
           const double *diag_inv, const double *b_glob, double *x_glob, double tol, int maxit,
           double *err_out);

/* diagonal of the element Helmholtz matrices, by applying the operator to unit
 * vectors (the reference assembles it from dense local matrices,
 * PreconditionerDiagonal.cpp:93-125); out has nelmt*ncoef entries. */
void or_helmholtz_diag(const or_helm_desc *h, double *out);

#ifdef __cplusplus
}
#endif
#endif
