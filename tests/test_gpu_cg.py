"""Global Helmholtz solve on the device (GlobalLinSysIterativeFull + diagonal
preconditioner + NekLinSysIterCG) against the oracle's CG, and against a
manufactured solution."""
import numpy as np
import pytest

import nektar_b200 as nb
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _system(n, nm, amp, lam=1.0):
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=amp, coords=True)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(lam)
    return m, op, nb.GlobalLinSys([op], gmap, nglob, ndir), gmap, nglob, ndir


def test_diagonal_preconditioner_matches_oracle():
    m, op, S, gmap, nglob, ndir = _system(3, 4, 0.05, 1.0)
    T = dict(m.T)
    T["w"] = m.T["ws"]
    dloc = O.helmholtz_diag("hex", m.nm, m.nq, m.nelmt, T, m.jac, m.df, 1.0, True)
    dinv = 1.0 / O.assemble(gmap, None, dloc, nglob)[ndir:]
    assert rel_l2(S.diag_inv(), dinv) < 1e-12


@pytest.mark.parametrize("n,nm", [(3, 4), (4, 5)])
def test_cg_matches_oracle_cg(n, nm):
    lam = 1.0
    m, op, S, gmap, nglob, ndir = _system(n, nm, 0.05, lam)
    rng = np.random.default_rng(n)
    b_loc = rng.uniform(-1, 1, m.nelmt * m.nc)
    x_loc, rep = S.solve(b_loc, tol=1e-10, check_interval=4)
    assert rep.converged and rep.rel_residual < 1e-10
    T = dict(m.T)
    T["w"] = m.T["ws"]
    b_glob = O.assemble(gmap, None, b_loc, nglob)
    dinv = S.diag_inv()
    x_o, it_o, err_o = O.pcg("hex", nm, m.nq, m.nelmt, T, m.jac, m.df, lam, True, nglob, ndir,
                             gmap, None, dinv, b_glob, tol=1e-10)
    assert abs(rep.iterations - it_o) <= max(3, int(0.03 * it_o)), (rep.iterations, it_o)
    assert rel_l2(x_loc, O.global_to_local(gmap, None, x_o)) < 1e-9
    x_loc2, _ = S.solve(b_loc, tol=1e-13, check_interval=8)
    x_o2, _, _ = O.pcg("hex", nm, m.nq, m.nelmt, T, m.jac, m.df, lam, True, nglob, ndir, gmap,
                       None, dinv, b_glob, tol=1e-13)
    assert rel_l2(x_loc2, O.global_to_local(gmap, None, x_o2)) < 1e-11


def test_cg_graph_and_direct_launch_agree_bitwise():
    m, op, S, gmap, nglob, ndir = _system(3, 4, 0.05)
    b = np.random.default_rng(7).uniform(-1, 1, m.nelmt * m.nc)
    x1, r1 = S.solve(b, tol=1e-10, use_graph=True, check_interval=5)
    x2, r2 = S.solve(b, tol=1e-10, use_graph=False, check_interval=3)
    assert r1.iterations == r2.iterations
    assert np.array_equal(x1, x2)  # deterministic reductions, no atomics


def test_manufactured_solution():
    """-lap u + lambda u = f, u = sin(pi x) sin(pi y) sin(pi z) on the curved
    unit cube (the map fixes the boundary, so the Dirichlet data are zero).
    Nektar solves L + lambda M with RHS -(g, phi) for forcing g = -f
    (ContField.cpp:813-816), i.e. the local RHS is IProductWRTBase(f)."""
    lam = 1.0
    errs = []
    for nm in (4, 6):
        m, op, S, gmap, nglob, ndir = _system(3, nm, 0.05, lam)
        x, y, z = m.xyz
        u = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        f = (3 * np.pi ** 2 + lam) * u
        b_loc = nb.Operator("iproduct", m)(f)
        c_loc, rep = S.solve(b_loc, tol=1e-12)
        uh = nb.Operator("bwdtrans", m)(c_loc)
        errs.append(np.sqrt(np.mean((uh - u) ** 2)))
    assert errs[0] < 2e-3 and errs[1] < errs[0] / 20, errs


def test_maxit_is_reported():
    m, op, S, gmap, nglob, ndir = _system(3, 4, 0.05)
    b = np.random.default_rng(2).uniform(-1, 1, m.nelmt * m.nc)
    with pytest.raises(nb.NektarB200Error) as e:
        S.solve(b, tol=1e-14, maxit=5)
    assert e.value.code == nb.C.NKB_ERR_NOT_CONVERGED


def _mixed_system(n, nm, amp, lam=1.0):
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=amp, coords=True)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(lam)
    op32 = nb.Operator("helmholtz", m, precision="fp32")
    op32.set_factors(lam)
    S = nb.GlobalLinSys([op], gmap, nglob, ndir, ops32=[op32])
    return m, S, (op, op32)


@pytest.mark.parametrize("n,nm,delta", [(3, 5, 0.1), (4, 9, 0.1), (4, 7, 0.01)])
def test_mixed_precision_reliable_updates_match_fp64(n, nm, delta):
    """FP32 CG with FP64 reliable updates reaches the FP64 residual criterion
    (checked on the FP64 residual), its solution matches the FP64 solve, and
    keeping the search direction across updates keeps the iteration count
    near the FP64 one."""
    m, S, keep = _mixed_system(n, nm, 0.05)
    b = np.random.default_rng(n).uniform(-1, 1, m.nelmt * m.nc)
    x64, r64 = S.solve(b, tol=1e-12)
    xm, rm = S.solve(b, tol=1e-12, mixed=True, inner_tol=delta)
    assert rm.converged and rm.rel_residual < 1e-12 and rm.outer_iterations >= 2
    assert rel_l2(xm, x64) < 1e-10, rel_l2(xm, x64)
    # Krylov-preserving updates keep the FP64 count; restarts after drift
    # (high order, high condition number) cost at most about twice it
    bound = 1.3 * r64.iterations + 10 if rm.restarts == 0 else 2.2 * r64.iterations + 20
    assert rm.iterations <= bound, (rm.iterations, r64.iterations, rm.restarts)


def test_mixed_not_converged_reports_maxit():
    m, S, keep = _mixed_system(3, 5, 0.05)
    b = np.random.default_rng(1).uniform(-1, 1, m.nelmt * m.nc)
    with pytest.raises(nb.NektarB200Error) as e:
        S.solve(b, tol=1e-14, maxit=5, mixed=True)
    assert e.value.code == nb.C.NKB_ERR_NOT_CONVERGED


def test_mixed_requires_fp32_operators():
    m, op, S, gmap, nglob, ndir = _system(2, 4, 0.05)
    b = np.ones(m.nelmt * m.nc)
    with pytest.raises(nb.NektarB200Error) as e:
        S.solve(b, mixed=True)
    assert e.value.code == nb.C.NKB_ERR_INVALID


def test_sharded_solve_on_device_operators_matches_global_linsys():
    """The sharded solve with one rank and the device Helmholtz operator as
    its element operator gives the device CG's solution."""
    from oracle import oracle as O
    from nektar_b200.sharded import ShardedSystem, device_apply, partition
    m = nb.BoxMesh("hex", 4, 6, 7, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    nt, nc = m.nt, m.nc
    T = dict(m.T)
    T["w"] = m.T["ws"]

    def factory(lo, hi):
        op = nb.Operator("helmholtz", shape="hex", nm=6, nq=m.nq, nelmt=hi - lo, T=m.T,
                         jac=m.jac[lo * nt:hi * nt],
                         df=np.ascontiguousarray(m.df[:, lo * nt:hi * nt]), deformed=True)
        op.set_factors(1.0)
        return op

    lo, hi = partition(m.nelmt, 1, 0)
    diag = O.helmholtz_diag("hex", 6, m.nq, m.nelmt, T, m.jac, m.df, 1.0, True)
    S = ShardedSystem(gmap, None, nc, ndir, lo, hi, device_apply(factory, lo, hi), diag)
    b = np.random.default_rng(8).uniform(-1, 1, m.nelmt * nc)
    x, it = S.solve(b, np.zeros_like(b), tol=1e-12)
    op = factory(0, m.nelmt)
    xg, rep = nb.GlobalLinSys([op], gmap, nglob, ndir).solve(b, tol=1e-12)
    assert rel_l2(x, xg) < 1e-9


def test_all_dirichlet_system_returns_the_dirichlet_values():
    """A system whose every dof is Dirichlet (one linear hexahedron: no
    interior modes) has nothing to solve (GlobalLinSysStaticCond /
    IterativeFull return at once when nGlobDofs - nDirBndDofs == 0): the
    solve returns the local Dirichlet values after zero iterations."""
    m = nb.BoxMesh("hex", 1, 2, 3, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    assert nglob == ndir
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    S = nb.GlobalLinSys([op], gmap, nglob, ndir)
    rng = np.random.default_rng(4)
    xd = rng.uniform(-1, 1, nglob)
    x0 = xd[np.asarray(gmap)]
    x, rep = S.solve(rng.uniform(-1, 1, m.nelmt * m.nc), x0, tol=1e-12)
    S.close()
    op.close()
    assert rep.converged and rep.iterations == 0
    assert np.array_equal(x, x0)
