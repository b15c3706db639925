"""CUDA element operators (through the C ABI) against the reference's own
kernels (golden fixtures) and the oracle. FP64 bar: relative L2 <= 1e-12;
FP32 operators: relative L2 <= 2e-5."""
import numpy as np
import pytest

import nektar_b200 as nb
from oracle import oracle as O
from tests.helpers import golden_cases, load_case, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _op(optype, g, precision="fp64"):
    T = g["T"]
    return nb.Operator(optype, shape=g["shape"], nm=int(g["nm"]),
                       nq=tuple(int(v) for v in g["nq"]), nelmt=int(g["ne"]), T=T, jac=g["jac"],
                       df=g["df"], deformed=bool(g["deformed"]), precision=precision)


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.split("/")[-1][:-4])
def test_ops_match_reference_golden(path):
    g = load_case(path)
    assert rel_l2(_op("bwdtrans", g)(g["x_rand"]), g["out_bwdtrans"]) < TOL64
    assert rel_l2(_op("iproduct", g)(g["f"]), g["out_iproduct"]) < TOL64
    d = _op("physderiv", g)(g["f"])
    assert rel_l2(np.stack(d), g["out_physderiv"]) < TOL64
    assert rel_l2(_op("iproduct_deriv", g)(g["f3"]), g["out_iproduct_deriv"]) < TOL64
    adr = _op("linear_adr", g)
    adr.set_factors(float(g["lam"]))
    n = g["vel"].size // 3
    adr.set_varcoeffs(g["vel"][:n], g["vel"][n:2 * n], g["vel"][2 * n:])
    assert rel_l2(adr(g["x"]), g["out_linear_adr"]) < TOL64
    op = _op("helmholtz", g)
    op.set_factors(float(g["lam"]))
    assert rel_l2(op(g["x"]), g["out_helmholtz"]) < TOL64
    op.set_factors(float(g["lam"]), nb.DIFF_CONST, g["diff"])
    assert rel_l2(op(g["x"]), g["out_helmholtz_constdiff"]) < TOL64
    op.set_factors(float(g["lam"]), nb.DIFF_VAR, g["diff"])
    assert rel_l2(op(g["x"]), g["out_helmholtz_vardiff"]) < TOL64
    # back to identity diffusion: the packed metric is rebuilt
    op.set_factors(float(g["lam"]))
    assert rel_l2(op(g["x"]), g["out_helmholtz"]) < TOL64


def _oracle_T(m):
    T = dict(m.T)
    T["w"] = m.T["ws"]
    return T


@pytest.mark.parametrize("shape,n,nm,amp", [
    ("hex", 8, 5, 0.0),      # the 8^3 affine P=4 / Q=6 operator configuration
    ("hex", 5, 7, 0.05),     # curved P=6 / Q=8
    ("hex", 3, 9, 0.05),     # curved P=8 / Q=10
    ("prism", 4, 5, 0.05),
    ("tet", 3, 5, 0.05),
    ("tet", 2, 11, 0.05),    # P=10
])
def test_ops_match_oracle(shape, n, nm, amp):
    m = nb.BoxMesh(shape, n, nm, nm + 1, amp=amp)
    rng = np.random.default_rng(n * 100 + nm)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    f = rng.uniform(-1, 1, m.nelmt * m.nt)
    To = _oracle_T(m)
    dfm = m.deformed
    assert rel_l2(nb.Operator("bwdtrans", m)(x), O.bwdtrans(shape, nm, m.nq, m.nelmt, To["b"], x)) < TOL64
    assert rel_l2(nb.Operator("iproduct", m)(f),
                  O.iproduct(shape, nm, m.nq, m.nelmt, To["b"], To["w"], m.jac, f, dfm)) < TOL64
    d = nb.Operator("physderiv", m)(f)
    do = O.physderiv(shape, m.nq, m.nelmt, To["D"], To["z"], m.df, f, dfm)
    assert rel_l2(np.stack(d), np.stack(do)) < TOL64
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    yo = O.helmholtz(shape, nm, m.nq, m.nelmt, To, m.jac, m.df, x, 1.0, dfm)
    assert rel_l2(op(x), yo) < TOL64
    f3 = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    yo = O.iproduct_deriv(shape, nm, m.nq, m.nelmt, To, m.jac, m.df, f3, dfm)
    assert rel_l2(nb.Operator("iproduct_deriv", m)(f3), yo) < TOL64
    vel = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    yo = O.linear_adr(shape, nm, m.nq, m.nelmt, To, m.jac, m.df, 0.7, vel, x, dfm)
    adr = nb.Operator("linear_adr", m)
    adr.set_factors(0.7)
    n = m.nelmt * m.nt
    adr.set_varcoeffs(vel[:n], vel[n:2 * n], vel[2 * n:])
    assert rel_l2(adr(x), yo) < TOL64


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_fp32_ops_match_oracle(shape):
    import torch
    m = nb.BoxMesh(shape, 3, 6, 7, amp=0.05)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    To = _oracle_T(m)
    yo = O.helmholtz(shape, m.nm, m.nq, m.nelmt, To, m.jac, m.df, x, 2.0, True)
    op = nb.Operator("helmholtz", m, precision="fp32")
    op.set_factors(2.0)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.empty(m.nelmt * m.nc, dtype=torch.float32, device="cuda")
    op.apply_device(xd.data_ptr(), yd.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel_l2(yd.double().cpu().numpy(), yo) < TOL32


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_helmholtz_diagonal_matches_oracle(shape):
    m = nb.BoxMesh(shape, 2, 4, 5, amp=0.05)
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.3)
    dg = op.helmholtz_diag()
    do = O.helmholtz_diag(shape, m.nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, 1.3, True)
    assert rel_l2(dg, do) < TOL64


def test_device_pointer_path_matches_host_path():
    import torch
    m = nb.BoxMesh("hex", 4, 5, 6, amp=0.05)
    op = nb.Operator("helmholtz", m)
    x = np.random.default_rng(1).uniform(-1, 1, m.nelmt * m.nc)
    yh = op(x)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    s = torch.cuda.Stream()
    op.apply_device(xd.data_ptr(), yd.data_ptr(), stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(yd.cpu().numpy(), yh)  # same kernel, same order: bitwise


@pytest.mark.parametrize("n,nm", [(1, 5), (3, 7), (2, 9), (1, 11), (5, 2)])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 6, 7, 8])
def test_tuned_and_generic_hex_helmholtz_agree(monkeypatch, n, nm, variant):
    """Every variant of the tuned Hex kernel (nkb_hex.cu: TMA-staged or
    streamed geometry, 1-2 elements per CTA, FP64 tensor cores for nq <= 8)
    against the shape-generic kernel, odd element counts included (partially
    filled last CTA)."""
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05)
    x = np.random.default_rng(nm).uniform(-1, 1, m.nelmt * m.nc)
    monkeypatch.setenv("NKB_HEX_VARIANT", str(variant))
    tuned = nb.Operator("helmholtz", m)
    tuned.set_factors(0.3)
    monkeypatch.setenv("NKB_KERNEL", "generic")
    generic = nb.Operator("helmholtz", m)
    generic.set_factors(0.3)
    assert rel_l2(tuned(x), generic(x)) < 1e-13


@pytest.mark.parametrize("n,nm", [(1, 5), (3, 7), (2, 9), (1, 11), (5, 2)])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 6, 7, 8])
def test_hex_kernel_variants_linear_adr_match_oracle(monkeypatch, n, nm, variant):
    """LinearADR through every variant of the tuned Hex kernel (its advection
    mode) against the oracle; a variant without room for the three extra
    geometry rows falls back to the generic kernel."""
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05)
    rng = np.random.default_rng(nm + 100)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    vel = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    k = m.nelmt * m.nt
    monkeypatch.setenv("NKB_HEX_VARIANT", str(variant))
    op = nb.Operator("linear_adr", m)
    op.set_factors(0.6)
    op.set_varcoeffs(vel[:k], vel[k:2 * k], vel[2 * k:])
    yo = O.linear_adr("hex", nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, 0.6, vel, x, True)
    assert rel_l2(op(x), yo) < TOL64


@pytest.mark.parametrize("shape,nm", [("prism", 3), ("prism", 7), ("prism", 11), ("tet", 4),
                                      ("tet", 8), ("tet", 11)])
def test_column_kernel_linear_adr_matches_oracle(shape, nm):
    m = nb.BoxMesh(shape, 2, nm, nm + 1, amp=0.05)
    rng = np.random.default_rng(nm + 200)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    vel = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    k = m.nelmt * m.nt
    op = nb.Operator("linear_adr", m)
    assert op.kernel().startswith("k_col_helm")
    op.set_factors(-2.0)
    op.set_varcoeffs(vel[:k], vel[k:2 * k], vel[2 * k:])
    yo = O.linear_adr(shape, nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, -2.0, vel, x, True)
    assert rel_l2(op(x), yo) < TOL64


@pytest.mark.parametrize("shape,n,nm", [("prism", 2, 4), ("tet", 2, 5), ("prism", 1, 9), ("tet", 1, 11)])
def test_static_and_runtime_size_generic_helmholtz_agree(monkeypatch, shape, n, nm):
    """Prism / Tet Helmholtz with compile-time sizes against the same kernel
    with run-time sizes."""
    m = nb.BoxMesh(shape, n, nm, nm + 1, amp=0.05)
    x = np.random.default_rng(nm).uniform(-1, 1, m.nelmt * m.nc)
    monkeypatch.setenv("NKB_COL", "0")
    fast = nb.Operator("helmholtz", m)
    fast.set_factors(0.7)
    y_fast = fast(x)  # the switches are read at launch time
    monkeypatch.setenv("NKB_GENERIC_STATIC", "0")
    slow = nb.Operator("helmholtz", m)
    slow.set_factors(0.7)
    assert rel_l2(y_fast, slow(x)) < 1e-13


@pytest.mark.parametrize("shape,n,nm", [("prism", 2, 3), ("prism", 1, 8), ("prism", 1, 11),
                                        ("tet", 2, 4), ("tet", 1, 7), ("tet", 1, 11)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_column_and_generic_helmholtz_agree(monkeypatch, shape, n, nm, precision, tol):
    """Prism / Tet column kernels (k direction in registers) against the
    shape-generic kernel."""
    import torch
    m = nb.BoxMesh(shape, n, nm, nm + 1, amp=0.05)
    x = np.random.default_rng(nm).uniform(-1, 1, m.nelmt * m.nc)
    dt = torch.float64 if precision == "fp64" else torch.float32
    xd = torch.tensor(x, dtype=dt, device="cuda")

    def apply(op):
        yd = torch.empty(m.nelmt * m.nc, dtype=dt, device="cuda")
        op.apply_device(xd.data_ptr(), yd.data_ptr(),
                        stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return yd.double().cpu().numpy()

    col = nb.Operator("helmholtz", m, precision=precision)
    col.set_factors(1.3)
    y_col = apply(col)  # the switch is read at launch time
    monkeypatch.setenv("NKB_COL", "0")
    gen = nb.Operator("helmholtz", m, precision=precision)
    gen.set_factors(1.3)
    assert rel_l2(y_col, apply(gen)) < tol


@pytest.mark.parametrize("shape", ["prism", "tet"])
def test_column_kernel_gathered_in_cg(monkeypatch, shape):
    """The column kernels' gathered form (inside the CG): a block-diagonal
    system (every local dof its own global dof) solved with the column and
    with the generic kernels."""
    m = nb.BoxMesh(shape, 2, 5, 6, amp=0.05)
    nloc = m.nelmt * m.nc
    gmap = np.arange(nloc, dtype=np.int32)
    b = np.random.default_rng(4).uniform(-1, 1, nloc)
    op = nb.Operator("helmholtz", m)
    op.set_factors(2.0)
    S = nb.GlobalLinSys([op], gmap, nloc, 0)
    xa, ra = S.solve(b, tol=1e-12)
    monkeypatch.setenv("NKB_COL", "0")
    op2 = nb.Operator("helmholtz", m)
    op2.set_factors(2.0)
    S2 = nb.GlobalLinSys([op2], gmap, nloc, 0)
    xb, rb = S2.solve(b, tol=1e-12)
    assert ra.converged and rb.converged
    assert rel_l2(xa, xb) < 1e-10


@pytest.mark.parametrize("shape,nm", [("hex", 7), ("prism", 6), ("tet", 9)])
def test_iproduct_deriv_three_array_forms_agree(shape, nm):
    """nkb_op_apply3 (three host arrays, three device arrays) and
    nkb_op_apply (one array holding the three fields) give one result."""
    import torch
    m = nb.BoxMesh(shape, 3, nm, nm + 1, amp=0.05)
    op = nb.Operator("iproduct_deriv", m)
    rng = np.random.default_rng(nm)
    f = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    n = m.nelmt * m.nt
    y = op(f)
    assert np.array_equal(op.apply3(f[:n], f[n:2 * n], f[2 * n:]), y)
    fd = [torch.tensor(f[k * n:(k + 1) * n], device="cuda") for k in (2, 0, 1)]
    yd = torch.empty(op.out_size, dtype=torch.float64, device="cuda")
    op.apply3_device(fd[1].data_ptr(), fd[2].data_ptr(), fd[0].data_ptr(), yd.data_ptr(),
                     stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), y)
    with pytest.raises(nb.NektarB200Error):
        nb.Operator("helmholtz", m).apply3_device(fd[0].data_ptr(), fd[1].data_ptr(),
                                                  fd[2].data_ptr(), yd.data_ptr())


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_fp32_iproduct_deriv_matches_oracle(shape):
    import torch
    m = nb.BoxMesh(shape, 3, 6, 7, amp=0.05)
    f = np.random.default_rng(9).uniform(-1, 1, 3 * m.nelmt * m.nt)
    yo = O.iproduct_deriv(shape, m.nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, f, True)
    op = nb.Operator("iproduct_deriv", m, precision="fp32")
    fd = torch.tensor(f, dtype=torch.float32, device="cuda")
    yd = torch.empty(op.out_size, dtype=torch.float32, device="cuda")
    op.apply_device(fd.data_ptr(), yd.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel_l2(yd.double().cpu().numpy(), yo) < TOL32


@pytest.mark.parametrize("shape,n,nm", [("hex", 12, 7), ("prism", 8, 6), ("tet", 6, 6)])
def test_iproduct_deriv_of_gradient_is_laplacian(shape, n, nm):
    """Size-independent identity at larger sizes: the weak Laplacian of
    Helmholtz with lambda = 0 equals IProductWRTDerivBase applied to
    PhysDeriv(BwdTrans(x)) (same quadrature, same metric terms)."""
    m = nb.BoxMesh(shape, n, nm, nm + 1, amp=0.05)
    x = np.random.default_rng(n).uniform(-1, 1, m.nelmt * m.nc)
    u = nb.Operator("bwdtrans", m)(x)
    grad = nb.Operator("physderiv", m)(u)
    y = nb.Operator("iproduct_deriv", m)(np.concatenate(grad))
    lap = nb.Operator("helmholtz", m)
    lap.set_factors(0.0)
    assert rel_l2(y, lap(x)) < 1e-12


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_linear_adr_factor_semantics(shape):
    """The reference scales the velocities by -1/lambda when they are set
    (LinearAdvectionDiffusionReaction.cpp:662-672) and applies -lambda from
    the last UpdateFactors; zero velocity is minus the Helmholtz mass term."""
    import torch
    m = nb.BoxMesh(shape, 3, 5, 6, amp=0.05)
    To = _oracle_T(m)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    vel = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    n = m.nelmt * m.nt
    adr = nb.Operator("linear_adr", m)
    # before any velocities: -lambda M + L, lambda = 1 until set_factors
    h = nb.Operator("helmholtz", m)
    h.set_factors(-1.0)
    assert rel_l2(adr(x), h(x)) < TOL64
    # velocities scaled with lambda = 2, then lambda changed to 3: V' = -V/2
    adr.set_factors(2.0)
    vd = torch.tensor(vel, device="cuda")
    adr.set_varcoeffs(vd[:n].data_ptr(), vd[n:2 * n].data_ptr(), vd[2 * n:].data_ptr())
    adr.set_factors(3.0)
    yo = O.linear_adr(shape, m.nm, m.nq, m.nelmt, To, m.jac, m.df, 3.0, 1.5 * vel, x, True)
    assert rel_l2(adr(x), yo) < TOL64
    with pytest.raises(nb.NektarB200Error):
        adr.set_factors(1.0, nb.DIFF_CONST, np.ones(6))
    with pytest.raises(nb.NektarB200Error):
        h.set_varcoeffs(vel[:n], vel[n:2 * n], vel[2 * n:])


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_fp32_linear_adr_matches_oracle(shape):
    import torch
    m = nb.BoxMesh(shape, 3, 6, 7, amp=0.05)
    rng = np.random.default_rng(8)
    x = rng.uniform(-1, 1, m.nelmt * m.nc)
    vel = rng.uniform(-1, 1, 3 * m.nelmt * m.nt)
    n = m.nelmt * m.nt
    yo = O.linear_adr(shape, m.nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, 1.3, vel, x, True)
    op = nb.Operator("linear_adr", m, precision="fp32")
    op.set_factors(1.3)
    op.set_varcoeffs(vel[:n], vel[n:2 * n], vel[2 * n:])
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.empty(op.out_size, dtype=torch.float32, device="cuda")
    op.apply_device(xd.data_ptr(), yd.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel_l2(yd.double().cpu().numpy(), yo) < TOL32


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 6, 7, 8])
def test_hex_kernel_variants_are_repeatable(monkeypatch, variant):
    """Repeated applications of every Hex variant to one input give the same
    bits: a race between the warps of an element (a shared-memory store
    landing after another warp's copy) shows up as an occasional wrong
    element, which a one-shot comparison can miss."""
    m = nb.BoxMesh("hex", 16, 7, 8, amp=0.05)
    x = np.random.default_rng(11).uniform(-1, 1, m.nelmt * m.nc)
    monkeypatch.setenv("NKB_HEX_VARIANT", str(variant))
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    y0 = op(x)
    bad = sum(not np.array_equal(op(x), y0) for _ in range(150))
    assert bad == 0


@pytest.mark.parametrize("shape,n,nm,amp,coords", [("hex", 4, 7, 0.05, True), ("prism", 3, 5, 0.05, False),
                                                   ("tet", 3, 4, 0.0, True), ("hex", 3, 5, 0.0, False)])
def test_device_geometry_matches_host_geometry(shape, n, nm, amp, coords):
    """nkb_geom_fill_device: the host fill's arithmetic on the device (its
    sin / cos may round the last bit differently), curved and affine, with
    and without the point coordinates; an operator built from the device
    factors applies as the host-built one does."""
    mh = nb.BoxMesh(shape, n, nm, nm + 1, amp=amp, coords=coords)
    md = nb.BoxMesh(shape, n, nm, nm + 1, amp=amp, coords=coords, geom_device=0)
    for a, b in ((mh.jac, md.jac), (mh.df, md.df)) + (((mh.xyz, md.xyz),) if coords else ()):
        b = b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-14 * max(1.0, np.abs(a).max())
    x = np.random.default_rng(nm).uniform(-1, 1, mh.nelmt * mh.nc)
    oh = nb.Operator("helmholtz", mh)
    od = nb.Operator("helmholtz", md)
    for o in (oh, od):
        o.set_factors(1.3)
    assert rel_l2(od(x), oh(x)) < 1e-13


def test_peak_probe_rates_are_plausible():
    """nkb_peak_probe: the device's FP64 FMA, FP64 tensor-core MMA and FP32
    FMA rates (TFLOP/s) lie within the bounds a B200-class part can reach,
    FP32 above FP64; an unknown kind is rejected."""
    import ctypes
    rates = []
    for kind in (0, 1, 2):
        v = ctypes.c_double(0.0)
        nb.check(nb.lib().nkb_peak_probe(kind, 0, ctypes.byref(v)))
        rates.append(v.value)
    fma64, mma64, fma32 = rates
    assert 5.0 < fma64 < 100.0 and 5.0 < mma64 < 150.0 and 20.0 < fma32 < 250.0, rates
    assert fma32 > fma64, rates
    v = ctypes.c_double(0.0)
    assert nb.lib().nkb_peak_probe(3, 0, ctypes.byref(v)) == nb.C.NKB_ERR_INVALID


@pytest.mark.parametrize("shape,nm", [("hex", 4), ("hex", 7), ("prism", 5), ("tet", 6)])
def test_empty_collection_applies_as_a_no_op(shape, nm):
    """An operator over no elements (a rank or batch slot left without
    elements) is created and applied without launching anything."""
    m = nb.BoxMesh(shape, 1, nm, nm + 1, amp=0.05)
    op = nb.Operator("helmholtz", shape=shape, nm=nm, nq=m.nq, nelmt=0, T=m.T,
                     jac=m.jac[:0], df=np.ascontiguousarray(m.df[:, :0]), deformed=True)
    op.set_factors(1.0)
    assert op.in_size == 0 and op(np.zeros(0)).size == 0
    op.close()
