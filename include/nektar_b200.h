/*
 * nektar_b200.h -- C ABI of the B200 (sm_100a) matrix-free spectral/hp
 * element path: sum-factorised BwdTrans / IProductWRTBase / PhysDeriv /
 * Helmholtz operators for Hex, Prism and Tet collections, the C0 local <->
 * global assembly map, and the Jacobi-preconditioned conjugate-gradient solve
 * of GlobalLinSysIterativeFull.
 *
 * Plain C: pointers, sizes and int status codes; no exceptions and no torch
 * types cross this boundary. Every call returns NKB_OK (0) or a negative
 * status; nkb_last_error() gives a message for the calling thread.
 *
 * Numbering of shapes, operators, points and basis types is that of the
 * reference (LibUtilities::ShapeType, Collections::OperatorType,
 * LibUtilities::PointsType, LibUtilities::BasisType) so that an adaptor can
 * pass the reference's enums through unchanged.
 *
 * Array layouts are those of the reference's Collections layer:
 *   - per-element data contiguous and element-major: coefficients
 *     in[e*ncoeffs + m], physical values phys[e*nqtot + q], q = (k*nq1+j)*nq0+i;
 *   - coefficient order: Hex p fastest then q then r; Prism / Tet r fastest
 *     inside (p, q) with the triangular truncation of the Modified_B/C bases;
 *   - jac: CoalescedGeomData::GetJac (nelmt*nqtot deformed, nelmt regular);
 *   - df : CoalescedGeomData::GetDerivFactors, 9 rows of ncol (= nelmt*nqtot
 *          deformed, nelmt regular) values; row k*3+j holds d xi_j / d x_k;
 *   - bdata/dbdata: Basis::GetBdata / GetDbdata; w: Points weights (raw, the
 *     Radau factors of MatrixFree SetUpZW are applied inside); D: column-major
 *     collocation derivative D[k*nq+i] = d l_k/dz(z_i) (Points::GetD()).
 */
#ifndef NEKTAR_B200_H
#define NEKTAR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define NKB_OK 0
#define NKB_ERR_INVALID -1     /* bad argument (NULL, size, unsupported combo) */
#define NKB_ERR_UNSUPPORTED -2 /* valid request this build does not implement */
#define NKB_ERR_CUDA -3        /* a CUDA runtime call failed */
#define NKB_ERR_NOMEM -4       /* device or host allocation failed */
#define NKB_ERR_NOT_CONVERGED -5 /* CG reached maxit (reference: warning + return) */
#define NKB_ERR_NONFINITE -6   /* NaN/Inf detected in a CG scalar */
#define NKB_ERR_NO_DEVICE -7   /* no CUDA device visible */
#define NKB_ERR_TIMEOUT -8     /* a bounded device wait gave up: the outputs of the elements
                                  it guarded were not written (the context stays usable) */

/* ---- enums (reference numbering) ---------------------------------------- */
#define NKB_TET 5   /* LibUtilities::eTetrahedron */
#define NKB_PRISM 7 /* LibUtilities::ePrism */
#define NKB_HEX 8   /* LibUtilities::eHexahedron */

#define NKB_BWDTRANS 0  /* Collections::eBwdTrans */
#define NKB_HELMHOLTZ 1 /* Collections::eHelmholtz */
#define NKB_LINEAR_ADR 2 /* Collections::eLinearAdvectionDiffusionReaction */
#define NKB_IPRODUCT 3  /* Collections::eIProductWRTBase */
#define NKB_IPRODUCT_DERIV 4 /* Collections::eIProductWRTDerivBase */
#define NKB_PHYSDERIV 5 /* Collections::ePhysDeriv */
#define NKB_DENSE_BLOCK 64 /* per-element dense matrices (no Collections counterpart) */

#define NKB_GLL 4       /* LibUtilities::eGaussLobattoLegendre */
#define NKB_RADAU_A1 11 /* LibUtilities::eGaussRadauMAlpha1Beta0 */
#define NKB_RADAU_A2 12 /* LibUtilities::eGaussRadauMAlpha2Beta0 */

#define NKB_MODIFIED_A 4 /* LibUtilities::eModified_A */
#define NKB_MODIFIED_B 5 /* LibUtilities::eModified_B */
#define NKB_MODIFIED_C 6 /* LibUtilities::eModified_C */

/* arithmetic of an operator */
#define NKB_FP64 0
#define NKB_FP32 1

/* nkb_op_apply / nkb_cg_solve flags */
#define NKB_DEVICE_PTRS 0 /* arrays are device pointers; call is stream-ordered */
#define NKB_HOST_PTRS 1   /* arrays are host pointers; copies in/out, synchronous */

/* Helmholtz diffusion modes (Collections::Helmholtz_MatrixFree::UpdateFactors) */
#define NKB_DIFF_NONE 0  /* identity diffusion */
#define NKB_DIFF_CONST 1 /* eFactorCoeffD00..D22: constant anisotropic tensor */
#define NKB_DIFF_VAR 2   /* eFactorTau: per-point tensor (SetVarDiffusion) */

/* ---- library ------------------------------------------------------------ */

/* Message of the last failed call on this thread ("" if none). */
const char *nkb_last_error(void);

/* Build string (version, sm arch, CUDA runtime). */
const char *nkb_version(void);

/* ---- 1-D setup tables (FP64, host) ---------------------------------------
 * Replace what the reference gets from LibUtilities::PointsManager and
 * BasisManager (GaussPoints.cpp:79-240, Basis.cpp:466-644). Provided for
 * callers that do not run the reference's Foundations library. */

/* z, w (raw weights) and D (column-major, D[k*np+i] = l_k'(z_i)) of a points
 * type: NKB_GLL, NKB_RADAU_A1, NKB_RADAU_A2. */
int nkb_points(int ptype, int np, double *z, double *w, double *D);

/* bdata / dbdata of a modified basis (NKB_MODIFIED_A/B/C) with nm modes at
 * the np points z with derivative matrix D. Returns the number of tabulated
 * modes (nm, nm(nm+1)/2, nm(nm+1)(nm+2)/6) or a negative status. */
int nkb_basis(int btype, int nm, int np, const double *z, const double *D, double *bdata,
              double *dbdata);

/* ---- element operators ---------------------------------------------------
 * One operator = one reference Collection of nelmt elements of the same
 * shape, basis and geometry type, i.e. one Collections::Operator instance:
 *   Collections::Operator (Collections/Operator.h:137-245), constructed
 *   through OPERATOR_CREATE / GetOperatorFactory (Operator.h:43-54,118-129),
 *   implemented by Helmholtz_MatrixFree (Collections/Helmholtz.cpp:586-761),
 *   BwdTrans_MatrixFree (BwdTrans.cpp:160-243), IProductWRTBase_MatrixFree
 *   (IProductWRTBase.cpp:182-268), PhysDeriv_MatrixFree (PhysDeriv.cpp:272-),
 *   IProductWRTDerivBase_MatrixFree (IProductWRTDerivBase.cpp:276-374),
 *   LinearAdvectionDiffusionReaction_MatrixFree
 *   (LinearAdvectionDiffusionReaction.cpp:548-790).
 */
typedef struct nkb_op nkb_op;

typedef struct nkb_op_desc
{
    int shape;    /* NKB_HEX / NKB_PRISM / NKB_TET */
    int optype;   /* NKB_BWDTRANS / NKB_HELMHOLTZ / NKB_LINEAR_ADR / NKB_IPRODUCT /
                     NKB_IPRODUCT_DERIV / NKB_PHYSDERIV */
    int nm;       /* modes per direction, equal in all directions (bdata[i] holds
                     nm x nq[i] values); collections of per-direction orders, which the
                     reference's MatrixFree operators take through their run-time-sized
                     path (MatrixFreeOps/Helmholtz.h:374-384), are not representable and
                     stay on the reference's own implementation types */
    int nq[3];    /* points per direction (Tet: nq0, nq0-1, nq0-1; Prism: nq0, nq0, nq0-1) */
    int ptype[3]; /* points type per direction */
    int nelmt;    /* elements in the collection */
    int deformed; /* 1: geometry per quadrature point (eDeformed), 0: per element */
    /* host arrays, reference layouts (see top of file); NULL where the
     * operator does not need them: BwdTrans needs bdata; IProduct bdata, w, jac;
     * PhysDeriv z, D, df; Helmholtz, LinearADR and IProductWRTDerivBase
     * bdata, w, z, D, jac, df. jac and df may also be device memory (copied
     * device to device). */
    const double *bdata[3];
    const double *w[3];
    const double *z[3];
    const double *D[3];
    const double *jac;
    const double *df;
    int precision; /* NKB_FP64 or NKB_FP32 (FP32 storage and arithmetic) */
    int device;    /* CUDA device ordinal */
} nkb_op_desc;

/* Replaces OPERATOR_CREATE(...)::create + the MatrixFree constructors
 * (Helmholtz.cpp:713-760 etc.): uploads tables, packs the geometry. */
int nkb_op_create(const nkb_op_desc *desc, nkb_op **op);

/* Per-element dense operator y_e = M_e x_e: nelmt blocks of n x n FP64
 * matrices (host, row-major, element after element), e.g. the Schur
 * complements of a statically condensed Helmholtz system
 * (GlobalLinSysIterativeStaticCond.cpp). It applies, gathers and feeds a CG
 * system's Jacobi preconditioner (its diagonal) like a Helmholtz operator;
 * in and out are nelmt*n values. n <= 6144. */
int nkb_op_create_dense(int n, int nelmt, const double *mats, int device, nkb_op **op);

/* The same with rows x cols blocks (in nelmt*cols, out nelmt*rows values,
 * cols <= 6144): the per-element maps of a statically condensed solve around
 * its CG, i.e. the right-hand side condensation F_b - K_bi K_ii^-1 F_i and the
 * interior back substitution of GlobalLinSysStaticCond::v_Solve
 * (GlobalLinSysStaticCond.cpp:98-227), with a low-energy basis change folded
 * in. Not usable as a CG system's operator. */
int nkb_op_create_dense_rect(int rows, int cols, int nelmt, const double *mats, int device,
                             nkb_op **op);

/* Static condensation of per-element matrices on the device: the set-up of
 * GlobalLinSysIterativeStaticCond (GlobalLinSysIterativeStaticCond.cpp:199,
 * v_AssembleSchurComplement) and the per-element maps of
 * GlobalLinSysStaticCond::v_Solve (GlobalLinSysStaticCond.cpp:98-227). K
 * (device, nelmt x nc x nc, as nkb_op_element_matrices writes it) split by
 * the host index lists bm (nb >= 1 boundary modes) and im (ni >= 0 interior
 * modes, together a partition of the nc modes; im may be NULL when ni = 0);
 * R (host, nb x nb row-major, or
 * NULL for the identity) is the boundary transform (the low-energy basis).
 * Outputs (device): S = R (Kbb - Kbi Kii^-1 Kib) R^T (nelmt x nb x nb),
 * W (nelmt x nb x nc): W[:, bm] = R, W[:, im] = -R Kbi Kii^-1, and
 * V (nelmt x nc x (nb + ni)): V[bm, :nb] = R^T, V[im, :nb] = -Kii^-1 Kib R^T,
 * V[im, nb:] = Kii^-1. Kii is factored by Cholesky (NKB_ERR_INVALID if it
 * is not positive definite). Synchronous on `stream`. */
int nkb_condense(int nelmt, int nc, const double *K, int nb, const int *bm, int ni, const int *im,
                 const double *R, double *S, double *W, double *V, int device, void *stream);

/* Every element's matrix of an FP64 operator with as many outputs as inputs
 * per element (Helmholtz, LinearADR, square dense blocks): K[e][i][j] is
 * output i of element e for the unit input j, built on the device by nc
 * applications (what GlobalLinSys::v_GetBlock, GlobalLinSys.cpp:341-345,
 * asks the reference's element expansions for when it builds statically
 * condensed matrices). K holds nelmt * nc * nc doubles; flags as
 * nkb_op_apply. */
int nkb_op_element_matrices(nkb_op *op, double *K, int flags, void *stream);

/* Replaces Helmholtz_MatrixFree::UpdateFactors (Helmholtz.cpp:615-691):
 * lambda (eFactorLambda); diff_mode NKB_DIFF_CONST with diff =
 * (d00 d01 d11 d02 d12 d22) from eFactorCoeffD00..D22; NKB_DIFF_VAR fills the
 * per-point tensor with diff as SetVarDiffusion does under eFactorTau. */
int nkb_op_set_factors(nkb_op *op, double lambda, int diff_mode, const double *diff);
/* For NKB_LINEAR_ADR it replaces LinearAdvectionDiffusionReaction_MatrixFree::
 * UpdateFactors (LinearAdvectionDiffusionReaction.cpp:578-590): the operator
 * applies -lambda (SetLambda(-lambda)); diff_mode must be NKB_DIFF_NONE and
 * lambda nonzero. Until the first call lambda is 1. */

/* Replaces LinearAdvectionDiffusionReaction_MatrixFree::UpdateVarcoeffs
 * (LinearAdvectionDiffusionReaction.cpp:598-723): the advection velocities
 * eVarCoeffVelX/Y/Z, nelmt*ntot values each (host or device pointers per
 * flags), scaled by -1/lambda with the lambda of the last set_factors, as the
 * reference scales them when it copies them. So the operator is
 *   out = lambda' (phi, u + V'.grad u) + (grad phi, grad u),
 * lambda' = -lambda, V' = -V/lambda at the time of this call. Zero velocity
 * until the first call. Synchronous: returns when the packed operator data
 * are updated; with device pointers it first waits for all work on the
 * device (the arrays may be written on any stream). */
int nkb_op_set_varcoeffs(nkb_op *op, const double *velx, const double *vely, const double *velz,
                         int flags);

/* Replaces Collections::Operator::operator()(in, out0, out1, out2, wsp)
 * (Operator.h:148-152): out0 is overwritten (no accumulate); PhysDeriv
 * writes d/dx, d/dy, d/dz to out0, out1, out2; IProductWRTDerivBase reads
 * the three components of its vector field consecutively from in (component
 * c of element e at in + c*nelmt*ntot + e*ntot; nkb_op_apply3 takes them as
 * three arrays) and writes out0. flags: NKB_HOST_PTRS or
 * NKB_DEVICE_PTRS; stream: a cudaStream_t (NULL = the legacy default
 * stream), on which the kernel is enqueued. With
 * host pointers the result is in out0.. on return, as the reference's is. */
int nkb_op_apply(nkb_op *op, const double *in, double *out0, double *out1, double *out2,
                 int flags, void *stream);

/* Host-pointer apply that allocates no device memory. No counterpart in the
 * reference. nkb_op_apply with NKB_HOST_PTRS stages the arrays in device
 * memory it obtains with cudaMalloc; callers that may not allocate at this
 * point (a fixed device-memory budget reserved at start-up, or a time loop
 * that must not take the synchronisation cudaMalloc/cudaFree can cause) use
 * this instead: staging goes through one file-scope 32 MiB device array, so
 * the operator's input plus outputs must fit in 4 Mi doubles (larger ones
 * get NKB_ERR_INVALID). The first call on a device looks the array up
 * (cudaGetSymbolAddress); make it before capturing any stream. The call
 * makes the operator's device current and restores the caller's. All calls
 * share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. FP64 operators; synchronous, like the
 * NKB_HOST_PTRS path it mirrors. */
int nkb_op_apply_host_static(nkb_op *op, const double *in, double *out0, double *out1,
                             double *out2, void *stream);

/* IProductWRTDerivBase with its three input fields as separate arrays, as
 * IProductWRTDerivBase_MatrixFree::operator()(entry0, entry1, entry2, entry3)
 * takes them for a 3-D coordinate system (IProductWRTDerivBase.cpp:285-318):
 * out = sum_m (d phi / d x_m, in_m) for every mode phi. flags and stream as
 * nkb_op_apply. Only for NKB_IPRODUCT_DERIV operators. */
int nkb_op_apply3(nkb_op *op, const double *in0, const double *in1, const double *in2,
                  double *out, int flags, void *stream);

/* FP32 variant of nkb_op_apply for NKB_FP32 operators (device pointers). */
int nkb_op_apply_f32(nkb_op *op, const float *in, float *out0, float *out1, float *out2,
                     void *stream);

/* GetInputSize / GetOutputSize (Operator.h:178-226), per output array. */
int nkb_op_sizes(const nkb_op *op, long *in_size, long *out_size);

/* Diagonal of every element's Helmholtz matrix (nelmt*ncoeffs values, host
 * or device per flags), computed matrix-free on the device. The reference
 * builds it from dense element matrices (PreconditionerDiagonal.cpp:93-125). */
int nkb_op_helmholtz_diag(nkb_op *op, double *diag, int flags, void *stream);

/* Time in ms of the last nkb_op_apply's kernel on the device (CUDA events). */
int nkb_op_last_kernel_ms(const nkb_op *op, float *ms);

/* Status of the operator's device error word, read and cleared: NKB_OK, or
 * NKB_ERR_TIMEOUT when a bounded wait inside one of its kernels gave up since
 * the last check (the elements it guarded kept stale outputs). Call it once
 * the operator's work has completed, e.g. after synchronising the stream of
 * NKB_DEVICE_PTRS applies; host-pointer applies and CG solves check it
 * themselves. The reference's kernels run on the host and have no such
 * state; its ASSERTL0 on a failed apply is the nearest counterpart. */
int nkb_op_check_error(nkb_op *op);

/* Test hook: the number of polls after which a bounded wait inside the
 * operator's kernels gives up (0: at once; negative: the default, 2^24). A
 * wait that gives up records NKB_ERR_TIMEOUT and still waits (bounded) for
 * its copy or MMA to complete before the kernel exits. Used by the tests to
 * make the wait run out; no reference counterpart. */
int nkb_op_set_wait_limit(nkb_op *op, int polls);

/* Name of the device kernel the operator runs (the autotuned choice; gather =
 * 1: the one used when a system gathers its input through the map). For
 * reports; no reference counterpart. */
const char *nkb_op_kernel(const nkb_op *op, int gather);

void nkb_op_destroy(nkb_op *op);

/* Self-test of the fifth-generation tensor-core building blocks the FP32 Hex
 * Helmholtz kernel uses (no reference counterpart): D = A B for one 128-row
 * tile, A (128 x 8*ksteps, row-major, host) written into the kernel's
 * K-major operand forms as TF32 high and low parts: by its row writer
 * (column_writer = 0), its rotated column writer (1, dense layout) or its
 * column writer for the padded layout (2), B
 * (8*ksteps x n, row-major, host) in its K-major table form, n in {16, 32,
 * 64}; D (128 x n, host) read back from tensor memory. info[0]: the tensor
 * memory address, info[1]: 1 when the MMA completion wait succeeded. */
int nkb_tc_selftest(int column_writer, int n, int ksteps, const float *A, const float *B, float *D,
                    unsigned *info);

/* ---- batched application over many collections --------------------------
 * ExpList::GeneralMatrixOp (MultiRegions/ExpList.cpp:2666-2757) applies one
 * operator type collection by collection (one collection per shape and basis
 * key). nkb_batch does the same for a set of operators of one type in one
 * call: in/out are the concatenated per-collection local vectors in the
 * order given (PhysDeriv: each collection's three derivatives consecutively).
 * The collections run concurrently on nstreams streams (0: 4), largest first,
 * captured once as a CUDA graph per (in, out) pair. All operators of a batch
 * share one type and one precision; an FP32 batch is applied with
 * nkb_batch_apply_f32 (device pointers). */
typedef struct nkb_batch nkb_batch;
int nkb_batch_create(nkb_op *const *ops, int nops, int nstreams, nkb_batch **batch);
int nkb_batch_sizes(const nkb_batch *batch, long *in_size, long *out_size);
int nkb_batch_apply(nkb_batch *batch, const double *in, double *out, int flags, void *stream);
int nkb_batch_apply_f32(nkb_batch *batch, const float *in, float *out, void *stream);
/* device time of the last nkb_batch_apply (waits for it) */
int nkb_batch_last_ms(nkb_batch *batch, float *ms);
void nkb_batch_destroy(nkb_batch *batch);

/* ---- global system + CG --------------------------------------------------
 * One nkb_sys = GlobalLinSysIterativeFull with PreconditionerDiagonal over
 * an AssemblyMapCG (MultiRegions/GlobalLinSysIterativeFull.cpp:96-384,
 * PreconditionerDiagonal.cpp:93-189, AssemblyMap/AssemblyMapCG.cpp:2772-2906)
 * driving NekLinSysIterCG (LinearAlgebra/NekLinSysIterCG.cpp:118-372). */
typedef struct nkb_sys nkb_sys;

typedef struct nkb_sys_desc
{
    int nops;             /* Helmholtz operators (collections), in local-space order */
    nkb_op *const *ops;   /* FP64 Helmholtz (or NKB_DENSE_BLOCK) operators */
    nkb_op *const *ops32; /* optional FP32 twins for mixed precision (or NULL) */
    long nloc;            /* local coefficients = sum of nelmt*ncoeffs */
    int nglob;            /* global coefficients, Dirichlet ones first */
    int ndir;             /* Dirichlet global coefficients */
    const int *map;       /* host, nloc: local -> global (GetLocalToGlobalMap) */
    const double *sign;   /* host, nloc, or NULL when no sign change */
    int device;
} nkb_sys_desc;

typedef struct nkb_cg_opts
{
    double tol;         /* IterativeSolverTolerance (relative, default 1e-9) */
    int maxit;          /* NekLinSysMaxIterations (default 5000) */
    int check_interval; /* host convergence poll every k iterations (device
                           kernels stop updating once converged) */
    int use_graph;      /* capture the k-iteration block in a CUDA graph */
    int mixed;          /* 0: FP64 CG; 1: FP32 CG with FP64 reliable updates
                           (true residual b - Ax recomputed with the FP64
                           operators; needs ops32). Stops on the FP64
                           residual with the FP64 criterion. */
    double inner_tol;   /* mixed: FP32-residual reduction between reliable
                           updates (default 0.1, at most 0.5) */
    int max_outer;      /* mixed: maximum reliable updates (default 1000) */
} nkb_cg_opts;

typedef struct nkb_cg_report
{
    int iterations;       /* CG iterations (FP32 iterations for mixed) */
    int outer_iterations; /* mixed: reliable updates (FP64 residuals) */
    double rel_residual;  /* sqrt(eps / rhs_magnitude) as NekLinSysIterCG reports */
    int converged;
    double device_ms;     /* device time of the solve (CUDA events) */
    long kernel_launches; /* kernels of this library launched by the solve */
    int restarts;         /* mixed: FP32 recurrence restarts after drift */
} nkb_cg_report;

int nkb_sys_create(const nkb_sys_desc *desc, nkb_sys **sys);

/* GlobalLinSysIterativeFull::v_Solve with Dirichlet lifting: b_loc is the
 * local right-hand side (pLocInput), x_loc on input holds the Dirichlet
 * values in local layout (ContField::v_ImposeDirichletConditions) and zeros
 * elsewhere, on output the solution (pLocOutput). flags as nkb_op_apply.
 * The solve runs on `stream`, or on the system's own stream when it is NULL,
 * and returns once it has finished (the host polls convergence). */
int nkb_cg_solve(nkb_sys *sys, const double *b_loc, double *x_loc, const nkb_cg_opts *opts,
                 nkb_cg_report *report, int flags, void *stream);

/* The same solve without blocking (no reference counterpart: the serving
 * layer keeps many systems' solves in flight from one host thread).
 * nkb_cg_begin issues the lifting and the first direction and returns;
 * nkb_cg_poll advances the solve by at most one block of device work and
 * sets *done once the result is in x_loc (wait = 1: block until the pending
 * block has finished first); nkb_cg_end returns what nkb_cg_solve would
 * return and fills the report. b_loc/x_loc must stay valid until done.
 * Host pointers make the final poll synchronous. */
int nkb_cg_begin(nkb_sys *sys, const double *b_loc, double *x_loc, const nkb_cg_opts *opts,
                 int flags, void *stream);
int nkb_cg_poll(nkb_sys *sys, int wait, int *done);
int nkb_cg_end(nkb_sys *sys, nkb_cg_report *report);

/* A second system over the same operators, map and diagonal with its own
 * vectors and stream (concurrent solves of one mesh). */
int nkb_sys_clone(const nkb_sys *sys, nkb_sys **clone);

/* Helmholtz lambda of this system (overrides the operators' eFactorLambda for
 * its solves, Jacobi diagonal rebuilt from the split mass / Laplacian
 * diagonal, computed once per shared system). */
int nkb_sys_set_lambda(nkb_sys *sys, double lambda);

/* Block-Jacobi preconditioner: replaces PreconditionerBlock::v_DoPreconditioner
 * (MultiRegions/PreconditionerBlock.cpp:813-852) and the block step of
 * PreconditionerLowEnergy::v_DoPreconditioner (PreconditionerLowEnergy.cpp
 * :915-933). Block b covers the non-Dirichlet dofs bidx[bptr[b]..bptr[b+1])
 * (indices counted from the first non-Dirichlet dof, 1..256 per block, no
 * dof in two blocks); binv holds the blocks' inverses one after another, each
 * n*n doubles column-major (for the symmetric blocks of an SPD system either
 * order). Dofs outside every block keep the Jacobi step. bptr and bidx are
 * host arrays, binv host or device memory (nkb_blocks_invert's output), all
 * copied; set once per system, before any clone; FP64 solves only. */
int nkb_sys_set_blocks(nkb_sys *sys, int nblk, const int *bptr, const int *bidx,
                       const double *binv);

/* The entity blocks of the Block and LowEnergy preconditioners assembled on
 * the device from condensed element matrices already there (nkb_condense's
 * S; PreconditionerLowEnergy.cpp:568-760 gathers the same blocks on the
 * host). Blocks as nkb_sys_set_blocks' bptr (n_b = bptr[b+1] - bptr[b]
 * rows); A (device) holds the blocks one after another, n_b * n_b doubles
 * row-major each. Contribution c of block b (cptr[b] <= c < cptr[b+1], host
 * CSR) adds sign_i sign_j S[celm[c]][l_i][l_j] to A_b[i][j], l and sign the
 * n_b entries of cloc / csgn (host) that follow the earlier contributions';
 * S is nelmt x nbm x nbm (device). Contributions are added in their order
 * (the result does not depend on the launch). One call per collection, then
 * nkb_blocks_invert. Synchronous on `stream`. */
int nkb_blocks_accumulate(int nblk, const int *bptr, int ncontrib, const int *cptr,
                          const int *celm, const int *cloc, const signed char *csgn, int nelmt,
                          int nbm, const double *S, double *A, int device, void *stream);

/* Inverts every block of A (device, layout of nkb_blocks_accumulate) in
 * place; on return each block is its inverse column-major, as
 * nkb_sys_set_blocks takes it. Gauss-Jordan without pivoting: the blocks of
 * an SPD system; NKB_ERR_INVALID if a pivot is not positive. Synchronous on
 * `stream`. */
int nkb_blocks_invert(int nblk, const int *bptr, double *A, int device, void *stream);

/* Device bytes: shared by all clones (map, CSR, sign, split diagonal) and
 * owned by this instance (vectors, state, staging). Operators not included. */
int nkb_sys_footprint(const nkb_sys *sys, size_t *shared_bytes, size_t *instance_bytes);

/* AssemblyMapCG::Assemble / GlobalToLocal on device arrays. */
int nkb_sys_assemble(nkb_sys *sys, const double *loc, double *glob, void *stream);
int nkb_sys_global_to_local(nkb_sys *sys, const double *glob, double *loc, void *stream);

/* Local-space matvec y = A x (GeneralMatrixOp over all collections). */
int nkb_sys_matvec_local(nkb_sys *sys, const double *x_loc, double *y_loc, void *stream);

/* Inverse assembled diagonal (nglob - ndir entries) the preconditioner uses. */
int nkb_sys_diag_inv(nkb_sys *sys, double *diag_inv, int flags, void *stream);

/* Per-kernel device time of one CG iteration, averaged over `iters`
 * back-to-back launches of each kernel on the system's stream with the
 * current vectors (CUDA events): element operators with the fused gather,
 * assemble + (s,w) dot, update + preconditioner + (r,w),(r,r) dots, scalars.
 * No counterpart in the reference (its LIKWID regions time the same phases,
 * NekLinSysIterCG.cpp:207-276). */
typedef struct nkb_sys_profile
{
    double op_ms, assemble_ms, update_ms, scalars_ms;
    double op_bytes;    /* algorithmic bytes of one operator pass */
    double op_flops;    /* algorithmic flops of one operator pass */
} nkb_sys_profile;

int nkb_sys_profile_iteration(nkb_sys *sys, int iters, nkb_sys_profile *prof);

void nkb_sys_destroy(nkb_sys *sys);

/* ---- sharded solve ---------------------------------------------------------
 * The CG of GlobalLinSysIterativeFull + NekLinSysIterCG sharded by element
 * partition (MeshPartition.cpp:99), every vector on the device: per
 * iteration the shared dofs are summed across the shards
 * (AssemblyMapCG::UniversalAssemble, AssemblyMapCG.cpp:2894-2906) and the
 * three dot products in one all-reduce (NekLinSysIterCG.cpp:310). A shard is
 * an nkb_sys over its partition's elements whose global dofs are numbered
 *   [Dirichlet | free, this shard only (nint) | free shared, owned | free
 *   shared, owned by another shard]   (nown = nint + the owned shared ones)
 * A dof shared by several shards is owned by one of them (the lowest rank),
 * which alone counts it in dot products. */

/* NCCL communicator of a sharded solve: one rank per GPU. The library binds
 * libnccl.so.2 at the first call (the copy the process has loaded, else the
 * system's); NKB_ERR_UNSUPPORTED when there is none. A process that also
 * loads another NCCL under that name (torch does) must load it first.
 * Rank 0 makes the id (128 bytes), which the caller passes to every rank. */
typedef struct nkb_comm nkb_comm;
int nkb_comm_unique_id(unsigned char *id);
int nkb_comm_create(const unsigned char *id, int nranks, int rank, int device, nkb_comm **comm);
void nkb_comm_destroy(nkb_comm *comm);

typedef struct nkb_shard_plan
{
    int rank;                       /* this shard (0..nranks-1) */
    int nint;                       /* free dofs no other shard touches */
    int nown;                       /* free dofs this shard counts in dot products */
    const unsigned char *dir_owned; /* ndir flags: Dirichlet dofs this shard counts in |b|^2
                                       (NULL: all) */
    int nshared;                    /* dofs (Dirichlet or free) shared with other shards */
    const int *shared;              /* their indices in this shard's global numbering */
    const int *sptr;                /* nshared+1: the sources of each shared dof */
    const int *ssrc;                /* its sharing shards' values in rank order: -1 this
                                       shard's own, else a position in the receive buffer */
    int nnbr;                       /* shards that share dofs with this one */
    const int *nbr;                 /* their ranks, increasing */
    const int *nptr;                /* nnbr+1: each neighbour's slice of the send and the
                                       receive buffer */
    const int *nidx;                /* the dofs sent to each neighbour (this shard's numbering),
                                       in increasing mesh-wide global id: the neighbour's
                                       receive slice holds its values of the same dofs in the
                                       same order */
} nkb_shard_plan;

typedef struct nkb_shard_group nkb_shard_group;

/* A sharded system. With comm: this process's one shard (nlocal = 1,
 * plans[0].rank = the communicator's rank); exchanges by ncclSend/ncclRecv
 * with every neighbour in one NCCL group, the dot sums by one ncclAllReduce.
 * Without comm: nlocal shards of ranks 0..nlocal-1 in this process on one
 * device (the sharded recurrence on one GPU); exchanges by device copies.
 * The systems' Jacobi diagonals are summed at the shared dofs; from then on
 * the systems solve only through a group (FP64, Jacobi; no clones, blocks or
 * mixed precision), also after the group is destroyed. Host plan arrays,
 * copied. */
int nkb_shard_group_create(nkb_sys *const *systems, const nkb_shard_plan *plans, int nlocal,
                           nkb_comm *comm, nkb_shard_group **group);

/* One solve of every local shard (b_locs[i], x_locs[i] as nkb_cg_solve's
 * b_loc / x_loc of shard i; flags NKB_HOST_PTRS or NKB_DEVICE_PTRS);
 * synchronous. All shards hold the same iterations, residual and, at the
 * shared dofs, the same solution bits. */
int nkb_shard_group_solve(nkb_shard_group *group, const double *const *b_locs,
                          double *const *x_locs, const nkb_cg_opts *opts, nkb_cg_report *reps,
                          int flags);

/* Releases the group (before its communicator and its systems). */
void nkb_shard_group_destroy(nkb_shard_group *group);

/* ---- structured test meshes (FP64 setup, host) ---------------------------
 * Unit-cube box of n^3 cells, optionally curved by
 *   x' = x + amp * sin(pi x) sin(pi y) sin(pi z) in every coordinate,
 * with geometric factors from the analytic Jacobian at the quadrature points
 * of the given tables (no isoparametric interpolation). Cells are hexes, or
 * split into 2 prisms or 6 tets. Used by tests and benchmarks; a Nektar++
 * caller passes its own GeomFactors through nkb_op_desc instead. */
typedef struct nkb_geom_request
{
    int shape;        /* NKB_HEX / NKB_PRISM / NKB_TET */
    int n;            /* cells per direction */
    double amp;       /* curvature amplitude (0 = affine) */
    int ncells;       /* number of cells to use (<= n^3), or 0 for all */
    const int *cells; /* optional list of cell ids (x fastest) of length ncells */
    int nq[3];
    const double *z[3]; /* quadrature points per direction (collapsed for Tet/Prism) */
    int deformed;       /* 1: per-point factors, 0: one value per element */
} nkb_geom_request;

/* Arithmetic rate of the device measured in place, in TFLOP/s: kind 0 FP64
 * fused multiply-add on the CUDA cores, 1 FP64 tensor-core MMA (m8n8k4),
 * 2 FP32 fused multiply-add (independent chains per thread, the best of five
 * timed launches after three warm-up ones). The compute denominators of the
 * operators' rooflines; no counterpart in the reference. */
int nkb_peak_probe(int kind, int device, double *tflops);

/* Number of elements the request produces. */
long nkb_geom_nelmt(const nkb_geom_request *req);

/* Fill jac (nelmt*nqtot or nelmt) and df (9 rows of ncol) and, if xyz is not
 * NULL, the physical coordinates of every quadrature point (3 rows of
 * nelmt*nqtot). */
int nkb_geom_fill(const nkb_geom_request *req, double *jac, double *df, double *xyz);

/* The same into device memory (jac, df, xyz device pointers; req and its
 * arrays on the host), computed on the device: one thread per element and
 * point, the host fill's arithmetic with the device's sin / cos (the last
 * bit may differ). At most 32 points per direction. Synchronous on
 * `stream`. */
int nkb_geom_fill_device(const nkb_geom_request *req, double *jac, double *df, double *xyz,
                         int device, void *stream);

/* C0 assembly map for a hex box of n^3 elements with nm modes per direction
 * (Modified_A): boundary (Dirichlet) coefficients numbered first, as
 * AssemblyMapCG orders them. map has n^3*nm^3 entries; all signs are +1 for
 * this consistently oriented mesh. Returns nglob via *nglob and ndir. */
int nkb_hex_box_assembly(int n, int nm, int *map, int *nglob, int *ndir);

#ifdef __cplusplus
}
#endif
#endif /* NEKTAR_B200_H */
