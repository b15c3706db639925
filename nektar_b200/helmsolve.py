"""Helmholtz solve of a Nektar++ session on the B200 path, the sequence of
the reference's Helmholtz3D demo (library/Demos/MultiRegions/Helmholtz3D.cpp):

    forcing f at the quadrature points            (the "Forcing" function)
    b = -IProductWRTBase(f)                        (ContField::v_HelmSolve,
                                                    ContField.cpp:797-821)
    b += Neumann / Robin boundary inner products     (ContField.cpp:822-855)
    x = Dirichlet values (boundary-constrained projection), zero elsewhere
    solve (L + lambda M + Robin face mass) x = b with the lifting
                                                   (GlobalLinSysIterativeFull)
    u = BwdTrans(x)
    L_inf, L_2, H_1 errors against "ExactSolution" (ExpList::Linf / L2 / H1)

Every operator application and the CG run on the device through the C ABI
(nektar_b200.Operator, GlobalLinSys); the host reads the session, builds the
geometry, the assembly and the Dirichlet values, and evaluates the session's
functions at the quadrature points.

    python -m nektar_b200.helmsolve session.xml [--tol 1e-13] [--fld out.fld]
        [-I GlobalSysSoln=IterativeStaticCond] [-I Preconditioner=LowEnergyBlock]

The linear solver follows the session's SOLVERINFO (or -I overrides, as the
reference's command line takes them): GlobalSysSoln IterativeFull (the
default here) or IterativeStaticCond, Preconditioner Diagonal (default),
Block or LowEnergyBlock (static condensation only). The reference's direct
solvers (DirectFull, DirectStaticCond, ...) map to the iterative solve of the
same system, whose solution they share to the solver tolerance.
"""
import argparse
import json
import time
from dataclasses import dataclass

import numpy as np


@dataclass
class HelmResult:
    coeffs: np.ndarray  # local coefficients (element-major)
    phys: np.ndarray  # solution at the quadrature points
    iterations: int
    rel_residual: float
    converged: bool
    linf: float = None
    l2: float = None
    h1: float = None
    solve_ms: float = None


def errors(mesh, u, exact, device=0):
    """(L_inf, L_2, H_1) of u against exact at the quadrature points:
    ExpList::Linf, ExpList::L2 and ExpList::H1 (StdExpansion::L2 / H1 per
    element, integrals with the element's weights and Jacobian; H1 adds the
    squared L2 norms of the physical derivatives of u - exact)."""
    import nektar_b200 as nb
    d = u - exact
    W = mesh.quad_weights()
    linf = float(np.max(np.abs(d)))
    l2sq = float(np.sum(W * d * d))
    h1sq = l2sq
    for col, dc, Wc in zip(mesh.collections, mesh.split(d, "phys"), mesh.split(W, "phys")):
        for gr in nb.Operator("physderiv", col, device=device)(dc):
            h1sq += float(np.sum(Wc * gr * gr))
    return linf, float(np.sqrt(l2sq)), float(np.sqrt(h1sq))


SOLVERS = {"IterativeFull": "full", "DirectFull": "full", "XxtFull": "full", "PETScFull": "full",
           "IterativeStaticCond": "staticcond", "DirectStaticCond": "staticcond",
           "XxtStaticCond": "staticcond", "PETScStaticCond": "staticcond"}
# the multi-level variants condense the boundary system again over patches
# (GlobalLinSysStaticCond::v_Solve's next-level branch,
# GlobalLinSysStaticCond.cpp:190-205): the same discrete system, solved here
# by the one-level condensed CG (their regression records equal the one-level
# sessions', e.g. Helmholtz3D_CG_Hex_AllBCs_iter_ml.tst and _AllBCs.tst)
SOLVERS.update({k + "MultiLevelStaticCond": "staticcond"
                for k in ("Iterative", "Direct", "Xxt", "PETSc")})
PRECONS = {"Diagonal": "diagonal", "Block": "block", "LowEnergyBlock": "lowenergy"}


def linear_solver(solver_info):
    """(solver, preconditioner) of a session's SOLVERINFO: GlobalSysSoln and
    Preconditioner (MultiRegions GlobalLinSys / Preconditioner factories)."""
    sol = solver_info.get("GlobalSysSoln", "IterativeFull")
    pre = solver_info.get("Preconditioner", "Diagonal")
    if sol not in SOLVERS:
        raise ValueError("GlobalSysSoln %s is not supported" % sol)
    if pre not in PRECONS:
        raise ValueError("Preconditioner %s is not supported" % pre)
    solver, precon = SOLVERS[sol], PRECONS[pre]
    if solver == "full" and precon != "diagonal":
        raise ValueError("Preconditioner %s needs GlobalSysSoln IterativeStaticCond" % pre)
    return solver, precon


def helm_solve(session, device=0, tol=1e-12, maxit=5000, check_interval=16, raise_on_maxit=True,
               solver_info=None):
    """solver_info: overrides of the session's SOLVERINFO (GlobalSysSoln,
    Preconditioner)."""
    import nektar_b200 as nb
    from .meshgraph import SessionMesh
    info = dict(session.solver_info)
    info.update(solver_info or {})
    solver, precon = linear_solver(info)
    mesh = SessionMesh(session)
    if "Lambda" not in session.parameters:
        raise ValueError("the session defines no Lambda parameter")
    lam = float(session.parameters["Lambda"])
    forcing = session.function("Forcing")
    if forcing is None:
        raise ValueError("the session defines no Forcing function")
    f = forcing.evaluate(*mesh.xyz)
    cols = mesh.collections
    b_loc = -np.concatenate([nb.Operator("iproduct", c, device=device)(fc)
                             for c, fc in zip(cols, mesh.split(f, "phys"))])
    Hs = []
    for c in cols:
        H = nb.Operator("helmholtz", c, device=device)
        H.set_factors(lam)
        Hs.append(H)
    # Neumann / Robin: boundary inner products join the forcing, Robin face
    # mass matrices the operator
    rhs_w, robin = mesh.weak_terms()
    b_loc = b_loc + rhs_w
    x0 = mesh.dirichlet_local()
    nloc = mesh.nloc
    if solver == "full":
        # Robin blocks as extra per-face dense operators over the faces'
        # global dofs (GlobalLinSysIterativeFull::v_DoMatrixMultiply adds
        # AddRobinTraceContribution to the element operators)
        ops, gms, sgs, x0s, bs = list(Hs), [mesh.gmap], [mesh.sign], [x0], [b_loc]
        by_size = {}
        for dofs, M, loc in robin:
            by_size.setdefault(dofs.size, []).append((dofs, M, loc))
        for grp in by_size.values():
            ops.append(nb.DenseOperator(np.stack([M for _, M, _ in grp]), device=device))
            gms.append(np.concatenate([d for d, _, _ in grp]))
            sgs.append(np.ones(gms[-1].size))
            x0s.append(np.concatenate([mesh.sign[lc] * x0[lc] for _, _, lc in grp]))
            bs.append(np.zeros(gms[-1].size))
        S = nb.GlobalLinSys(ops, np.concatenate(gms), mesh.nglob, mesh.ndir,
                            sign=np.concatenate(sgs), device=device)
        b_sys, x0_sys = np.concatenate(bs), np.concatenate(x0s)
    else:
        from .staticcond import StaticCondSys, element_matrices
        K = [element_matrices(H) for H in Hs]
        for dofs, M, loc in robin:  # Expansion3D::v_AddRobinMassMatrix
            ci = int(np.searchsorted(mesh.offsets, loc[0], side="right")) - 1
            nc = mesh.collections[ci].nc
            el = int(loc[0] - mesh.offsets[ci]) // nc
            li = loc - mesh.offsets[ci] - el * nc
            sg = mesh.sign[loc]
            K[ci][el][np.ix_(li, li)] += np.outer(sg, sg) * M
        S = StaticCondSys(Hs, mesh.gmap, mesh.nglob, mesh.ndir, sign=mesh.sign, device=device,
                          matrices=K, precon=precon, lam=lam)
        b_sys, x0_sys = b_loc, x0
    t0 = time.perf_counter()
    x, rep = S.solve(b_sys, x0_sys, tol=tol, maxit=maxit, check_interval=check_interval,
                     raise_on_maxit=raise_on_maxit)
    x = x[:nloc]
    ms = (time.perf_counter() - t0) * 1e3
    u = np.concatenate([nb.Operator("bwdtrans", c, device=device)(xc)
                        for c, xc in zip(cols, mesh.split(x))])
    res = HelmResult(x, u, rep.iterations, rep.rel_residual, bool(rep.converged), solve_ms=ms)
    res.solver, res.precon = solver, precon
    exact = session.function("ExactSolution")
    if exact is not None:
        res.linf, res.l2, res.h1 = errors(mesh, u, exact.evaluate(*mesh.xyz), device)
    res.mesh = mesh
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("session")
    ap.add_argument("--tol", type=float, default=1e-12)
    ap.add_argument("--maxit", type=int, default=5000)
    ap.add_argument("--fld", default=None, help="write the solution as a .fld directory")
    ap.add_argument("--json", action="store_true")
    ap.add_argument("-I", dest="info", action="append", default=[],
                    help="SOLVERINFO override PROPERTY=VALUE")
    a = ap.parse_args()
    from .session import read_session
    s = read_session(a.session)
    over = dict(kv.split("=", 1) for kv in a.info)
    r = helm_solve(s, tol=a.tol, maxit=a.maxit, solver_info=over)
    if a.fld:
        from .fieldio import write_fld
        write_fld(a.fld, r.mesh, {"u": r.coeffs})
    if a.json:
        print(json.dumps({"session": s.name, "solver": r.solver, "precon": r.precon,
                          "iterations": r.iterations,
                          "rel_residual": r.rel_residual, "linf": r.linf, "l2": r.l2,
                          "h1": r.h1, "solve_ms": r.solve_ms}))
        return
    print("Solving 3D Helmholtz:")
    print("  - Lambda        : %g" % s.parameters["Lambda"])
    print("  - No. modes     : %s" % ",".join(str(c.nm) for c in r.mesh.collections))
    print("  - Solver        : %s, %s" % (r.solver, r.precon))
    print("  - CG iterations : %d (relative residual %.3g)" % (r.iterations, r.rel_residual))
    if r.l2 is not None:
        print("L infinity error: %g" % r.linf)
        print("L 2 error:        %g" % r.l2)
        print("H 1 error:        %g" % r.h1)


if __name__ == "__main__":
    main()
