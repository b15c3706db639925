"""The oracle (oracle/nkoracle.c, a plain-C restatement of the reference's
matrix-free kernels and CG) pinned against the reference's own kernels: the
committed golden fixtures (made by tests/golden/make_golden.py from the
reference sources compiled in place) and, where oracle/_ref is built, live
reference runs on fresh seeded inputs."""
import numpy as np
import pytest

from tests.helpers import golden_cases, load_case, rel_l2
from oracle import oracle as O
from oracle import ref

TOL = 1e-14  # same algorithm, same FP64 evaluation order up to fma contraction


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_matches_golden(path):
    g = load_case(path)
    s, nm, nq, ne, dfm = g["shape"], int(g["nm"]), tuple(int(v) for v in g["nq"]), int(g["ne"]), \
        bool(g["deformed"])
    T = dict(g["T"])
    T["w"] = T["ws"]  # the oracle takes SetUpZW-scaled weights
    y = O.bwdtrans(s, nm, nq, ne, T["b"], g["x_rand"])
    assert rel_l2(y, g["out_bwdtrans"]) < TOL
    y = O.iproduct(s, nm, nq, ne, T["b"], T["w"], g["jac"], g["f"], dfm)
    assert rel_l2(y, g["out_iproduct"]) < TOL
    d = O.physderiv(s, nq, ne, T["D"], T["z"], g["df"], g["f"], dfm)
    assert rel_l2(np.stack(d), g["out_physderiv"]) < TOL
    for mode, tag in ((0, "helmholtz"), (1, "helmholtz_constdiff"), (2, "helmholtz_vardiff")):
        y = O.helmholtz(s, nm, nq, ne, T, g["jac"], g["df"], g["x"], float(g["lam"]), dfm, mode,
                        g["diff"] if mode else None)
        assert rel_l2(y, g["out_" + tag]) < TOL, tag
    y = O.iproduct_deriv(s, nm, nq, ne, T, g["jac"], g["df"], g["f3"], dfm)
    assert rel_l2(y, g["out_iproduct_deriv"]) < TOL
    y = O.linear_adr(s, nm, nq, ne, T, g["jac"], g["df"], float(g["lam"]), g["vel"], g["x"], dfm)
    assert rel_l2(y, g["out_linear_adr"]) < TOL


def _tables(shape, nm, nq0):
    from tests.golden.make_golden import ref_tables
    return ref_tables(shape, nm, nq0)


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built (make -C oracle ref)")
@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
@pytest.mark.parametrize("nm", [4, 7])
def test_oracle_matches_live_reference(shape, nm):
    rng = np.random.default_rng(nm * 7 + len(shape))
    T, nq = _tables(shape, nm, nm + 1)
    ne, nt, nc = 9, nq[0] * nq[1] * nq[2], O.ncoeffs(shape, nm)
    jac = rng.uniform(0.5, 1.5, ne * nt)
    df = rng.uniform(-1, 1, (9, ne * nt))
    x = rng.uniform(-1, 1, ne * nc)
    To = dict(T)
    To["w"] = T["ws"]  # both take SetUpZW-scaled weights
    op = ref.RefOp(shape, "helmholtz", nm, nq, ne, To, jac=jac, df=df, deformed=True, nthreads=2)
    op.set_factors(0.7)
    y = np.zeros(ne * nc)
    op.apply(x, y)
    yo = O.helmholtz(shape, nm, nq, ne, To, jac, df, x, 0.7, True)
    assert rel_l2(yo, y) < TOL


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built (make -C oracle ref)")
@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
@pytest.mark.parametrize("deformed", [False, True])
def test_oracle_iproduct_deriv_matches_live_reference(shape, deformed):
    rng = np.random.default_rng(11 + len(shape) + deformed)
    nm = 6
    T, nq = _tables(shape, nm, nm + 1)
    ne, nt = 11, nq[0] * nq[1] * nq[2]
    ncol = ne * nt if deformed else ne
    jac = rng.uniform(0.5, 1.5, ncol)
    df = rng.uniform(-1, 1, (9, ncol))
    f = rng.uniform(-1, 1, 3 * ne * nt)
    To = dict(T)
    To["w"] = T["ws"]
    op = ref.RefOp(shape, "iproduct_deriv", nm, nq, ne, To, jac=jac, df=df, deformed=deformed,
                   nthreads=2)
    y = np.zeros(ne * O.ncoeffs(shape, nm))
    op.apply(f, y)
    yo = O.iproduct_deriv(shape, nm, nq, ne, To, jac, df, f, deformed)
    assert rel_l2(yo, y) < TOL


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built (make -C oracle ref)")
@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
@pytest.mark.parametrize("deformed", [False, True])
def test_oracle_linear_adr_matches_live_reference(shape, deformed):
    rng = np.random.default_rng(23 + len(shape) + deformed)
    nm = 5
    T, nq = _tables(shape, nm, nm + 1)
    ne, nt, nc = 10, nq[0] * nq[1] * nq[2], O.ncoeffs(shape, nm)
    ncol = ne * nt if deformed else ne
    jac = rng.uniform(0.5, 1.5, ncol)
    df = rng.uniform(-1, 1, (9, ncol))
    vel = rng.uniform(-1, 1, 3 * ne * nt)
    x = rng.uniform(-1, 1, ne * nc)
    To = dict(T)
    To["w"] = T["ws"]
    op = ref.RefOp(shape, "linear_adr", nm, nq, ne, To, jac=jac, df=df, deformed=deformed,
                   nthreads=2)
    op.set_adr(0.8, vel)
    y = np.zeros(ne * nc)
    op.apply(x, y)
    yo = O.linear_adr(shape, nm, nq, ne, To, jac, df, 0.8, vel, x, deformed)
    assert rel_l2(yo, y) < TOL
    # zero velocity: minus the Helmholtz operator's mass term plus its Laplacian
    op.set_adr(0.8, np.zeros_like(vel))
    op.apply(x, y)
    yh = O.helmholtz(shape, nm, nq, ne, To, jac, df, x, -0.8, deformed)
    assert rel_l2(y, yh) < TOL


def _hex_problem(n, nm, amp, lam):
    """Small curved hex box from the oracle's own view: tables from the
    reference Polylib, geometry and map from the product's setup routines
    (checked separately in test_setup.py)."""
    import nektar_b200 as nb
    mesh = nb.BoxMesh("hex", n, nm, nm + 1, amp=amp)
    gmap, nglob, ndir = mesh.assembly()
    T, nq = _tables("hex", nm, nm + 1)
    return mesh, T, nq, gmap, nglob, ndir


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built (make -C oracle ref)")
def test_oracle_cg_matches_reference_cg():
    n, nm, lam = 3, 4, 1.0
    mesh, T, nq, gmap, nglob, ndir = _hex_problem(n, nm, 0.05, lam)
    To = dict(T)
    To["w"] = T["ws"]
    rng = np.random.default_rng(3)
    nc = nm ** 3
    b_loc = rng.uniform(-1, 1, mesh.nelmt * nc)
    b_glob = O.assemble(gmap, None, b_loc, nglob)
    dloc = O.helmholtz_diag("hex", nm, nq, mesh.nelmt, To, mesh.jac, mesh.df, lam, True)
    dglob = O.assemble(gmap, None, dloc, nglob)
    dinv = 1.0 / dglob[ndir:]
    x_o, it_o, err_o = O.pcg("hex", nm, nq, mesh.nelmt, To, mesh.jac, mesh.df, lam, True, nglob,
                             ndir, gmap, None, dinv, b_glob, tol=1e-10)
    op = ref.RefOp("hex", "helmholtz", nm, nq, mesh.nelmt, To, jac=mesh.jac, df=mesh.df,
                   deformed=True)
    op.set_factors(lam)
    order = np.argsort(gmap, kind="stable")
    aptr = np.zeros(nglob + 1, dtype=np.int32)
    np.add.at(aptr, gmap + 1, 1)
    aptr = np.cumsum(aptr).astype(np.int32)
    x_r, it_r, err_r = ref.pcg_solve(nglob, ndir, gmap, None, aptr, order.astype(np.int64), op,
                                     dinv, b_glob, tol=1e-10)
    # CG near its stopping threshold is sensitive to the summation order of the
    # dot products (the reference driver sums per thread): allow 3 %
    assert abs(it_o - it_r) <= max(3, int(0.03 * it_r))
    assert err_o < 1e-10 and err_r < 1e-10
    # both stop at a relative residual of 1e-10; their solutions then differ by
    # at most the conditioning times that residual
    assert rel_l2(x_o, x_r) < 1e-9
    x_o2, _, _ = O.pcg("hex", nm, nq, mesh.nelmt, To, mesh.jac, mesh.df, lam, True, nglob, ndir,
                       gmap, None, dinv, b_glob, tol=1e-13)
    x_r2, _, _ = ref.pcg_solve(nglob, ndir, gmap, None, aptr, order.astype(np.int64), op, dinv,
                               b_glob, tol=1e-13)
    assert rel_l2(x_o2, x_r2) < 1e-11
