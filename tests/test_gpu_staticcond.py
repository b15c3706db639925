"""Static condensation on the device: the dense block kernel against numpy,
and the condensed solve against the full solve (curved hex box, mixed
hex/prism session with rotated frames and Dirichlet data)."""
import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200.staticcond import StaticCondSys
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_dense_operator_matches_numpy():
    rng = np.random.default_rng(0)
    mats = rng.uniform(-1, 1, (7, 218, 218))
    x = rng.uniform(-1, 1, 7 * 218)
    d = nb.DenseOperator(mats)
    y = d(x)
    ref = np.einsum("eij,ej->ei", mats, x.reshape(7, 218)).ravel()
    assert rel_l2(y, ref) < 1e-14
    assert d.kernel().startswith("k_dense_gemv")


def test_condensed_solve_matches_full_solve():
    m = nb.BoxMesh("hex", 4, 7, 8, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    b = np.random.default_rng(1).uniform(-1, 1, m.nelmt * m.nc)
    full = nb.GlobalLinSys([op], gmap, nglob, ndir)
    xf, rf = full.solve(b, tol=1e-12)
    sc = StaticCondSys([op], gmap, nglob, ndir)
    xs, rs = sc.solve(b, tol=1e-12)
    assert rel_l2(xs, xf) < 1e-9
    assert rs.iterations < rf.iterations


def test_condensed_solve_on_mixed_session():
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session, write_box_session
    U = "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    F = "-(Lambda + 3*PI*PI/4)*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    s = read_session(write_box_session("hexprism", 2, 5, 1.0, U, F, U, shuffle_seed=3))
    mesh = SessionMesh(s)
    ops = []
    for c in mesh.collections:
        H = nb.Operator("helmholtz", c)
        H.set_factors(1.0)
        ops.append(H)
    f = s.function("Forcing").evaluate(*mesh.xyz)
    b = -np.concatenate([nb.Operator("iproduct", c)(fc)
                         for c, fc in zip(mesh.collections, mesh.split(f, "phys"))])
    x0 = mesh.dirichlet_local()
    xf, _ = nb.GlobalLinSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, sign=mesh.sign).solve(
        b, x0, tol=1e-13)
    xs, _ = StaticCondSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, sign=mesh.sign).solve(
        b, x0, tol=1e-13)
    assert rel_l2(xs, xf) < 1e-9


@pytest.mark.parametrize("precon", ["block", "lowenergy"])
def test_block_and_lowenergy_preconditioned_solves(precon):
    m = nb.BoxMesh("hex", 4, 7, 8, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    b = np.random.default_rng(1).uniform(-1, 1, m.nelmt * m.nc)
    xf, rf = nb.GlobalLinSys([op], gmap, nglob, ndir).solve(b, tol=1e-12)
    xd, rd = StaticCondSys([op], gmap, nglob, ndir).solve(b, tol=1e-12)
    sc = StaticCondSys([op], gmap, nglob, ndir, precon=precon)
    assert sc.nblocks > 0
    xs, rs = sc.solve(b, tol=1e-12)
    assert rel_l2(xs, xf) < 1e-9
    if precon == "lowenergy":
        assert rs.iterations * 4 < rd.iterations
    else:
        assert rs.iterations < rd.iterations
    sc.close()


@pytest.mark.parametrize("shape", ["hex", "tet", "prism", "hexprism"])
def test_lowenergy_solve_on_sessions(shape):
    """Rotated element frames (signs in the map) and Dirichlet data, every
    shape and a hex/prism mesh: the low-energy condensed solve reproduces
    the full solve in a fraction of its iterations."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session, write_box_session, write_hex_box_session
    U = "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    F = "-(Lambda + 3*PI*PI/4)*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    if shape == "hex":
        s = read_session(write_hex_box_session(3, 6, 1.5, U, F, U, shuffle_seed=4))
    else:
        s = read_session(write_box_session(shape, 2, 6, 1.5, U, F, U, shuffle_seed=4))
    mesh = SessionMesh(s)
    ops = []
    for c in mesh.collections:
        H = nb.Operator("helmholtz", c)
        H.set_factors(1.5)
        ops.append(H)
    f = s.function("Forcing").evaluate(*mesh.xyz)
    b = -np.concatenate([nb.Operator("iproduct", c)(fc)
                         for c, fc in zip(mesh.collections, mesh.split(f, "phys"))])
    x0 = mesh.dirichlet_local()
    xf, rf = nb.GlobalLinSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, sign=mesh.sign).solve(
        b, x0, tol=1e-13)
    sc = StaticCondSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, sign=mesh.sign, precon="lowenergy")
    xs, rs = sc.solve(b, x0, tol=1e-13)
    assert rel_l2(xs, xf) < 1e-9
    assert rs.iterations * 3 < rf.iterations
    sc.close()


def test_set_blocks_rejects_bad_blocks():
    m = nb.BoxMesh("hex", 2, 4, 5, amp=0.0)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    sys_ = nb.GlobalLinSys([op], gmap, nglob, ndir)
    eye = np.eye(2)
    with pytest.raises(nb.NektarB200Error):  # a dof in two blocks
        sys_.set_blocks([(np.array([ndir, ndir + 1]), eye), (np.array([ndir + 1, ndir + 2]), eye)])
    with pytest.raises(nb.NektarB200Error):  # a Dirichlet dof
        sys_.set_blocks([(np.array([ndir - 1, ndir]), eye)])
    sys_.set_blocks([(np.array([ndir, ndir + 1]), eye)])
    with pytest.raises(nb.NektarB200Error):  # set twice
        sys_.set_blocks([(np.array([ndir + 2, ndir + 3]), eye)])
    # identity blocks on two dofs: still converges to the same solution
    b = np.random.default_rng(3).uniform(-1, 1, m.nelmt * m.nc)
    xb, _ = sys_.solve(b, tol=1e-12)
    xj, _ = nb.GlobalLinSys([op], gmap, nglob, ndir).solve(b, tol=1e-12)
    assert rel_l2(xb, xj) < 1e-9


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_element_matrices_on_device_match_unit_applications(shape):
    """nkb_op_element_matrices equals the operator applied to unit vectors
    one host call at a time, and is symmetric (a Helmholtz matrix)."""
    from nektar_b200.staticcond import element_matrices
    m = nb.BoxMesh(shape, 2, 5, 6, amp=0.05)
    op = nb.Operator("helmholtz", m)
    op.set_factors(0.7)
    K = element_matrices(op)
    nc, ne = m.nc, m.nelmt
    for j in (0, nc // 2, nc - 1):
        x = np.zeros(ne * nc)
        x[j::nc] = 1.0
        assert np.array_equal(K[:, :, j], op(x).reshape(ne, nc))
    assert np.abs(K - K.transpose(0, 2, 1)).max() < 1e-13 * np.abs(K).max()


def test_host_element_matrices_built_in_column_groups():
    """With host pointers nkb_op_element_matrices builds K a group of columns
    at a time in a device buffer of at most 1 GiB and copies each group into
    the strided host rows: at 12^3 P=6 (K = 1.6 GB, two groups) the host K
    equals the device-built one bit for bit."""
    import torch
    from nektar_b200.staticcond import element_matrices
    m = nb.BoxMesh("hex", 12, 7, 8, amp=0.05)
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    nc = m.nc
    assert m.nelmt * nc * nc * 8 > 2 ** 30
    Kh = element_matrices(op)
    Kd = torch.empty((m.nelmt, nc, nc), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    nb.check(nb.lib().nkb_op_element_matrices(op.h, Kd.data_ptr(), nb.DEVICE_PTRS, None))
    torch.cuda.synchronize()
    assert np.array_equal(Kh, Kd.cpu().numpy())
    op.close()


@pytest.mark.parametrize("shape,n,nm", [("hex", 3, 5), ("hex", 2, 7), ("prism", 2, 5),
                                        ("tet", 2, 4), ("hexprism", 2, 5), ("tet", 2, [3, 5, 4]),
                                        ("hexprism", 2, [5, 4])])
@pytest.mark.parametrize("precon", ["diagonal", "block", "lowenergy"])
def test_device_setup_matches_host_setup(shape, n, nm, precon):
    """The device set-up (element matrices kept on the device, nkb_condense:
    batched Cholesky, Schur complements and the W / V maps, the low-energy
    transform folded in; the Block / LowEnergy entity blocks accumulated
    and inverted there, nkb_blocks_accumulate / nkb_blocks_invert) gives the
    host set-up's condensed operators, preconditioned iterations and
    solutions; on meshes of variable order (nm a list of orders) the device
    condenses each group of elements that share a variable-order mask with
    its own masked transform."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session, with_orders, write_box_session
    U = "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    F = "-(Lambda + 3*PI*PI/4)*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
    orders = nm if isinstance(nm, list) else None
    nm = max(orders) if orders else nm
    txt = write_box_session(shape, n, nm - 1, 1.0, U, F, U, shuffle_seed=5)
    s = read_session(with_orders(txt, orders, seed=2) if orders else txt)
    mesh = SessionMesh(s)
    if orders:
        assert (mesh.sign == 0).any()
    ops = []
    for c in mesh.collections:
        H = nb.Operator("helmholtz", c)
        H.set_factors(1.0)
        ops.append(H)
    b = np.random.default_rng(nm).uniform(-1, 1, mesh.nloc)
    x0 = mesh.dirichlet_local()
    kw = dict(sign=mesh.sign, precon=precon, lam=1.0)
    host = StaticCondSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, setup="host", **kw)
    dev = StaticCondSys(ops, mesh.gmap, mesh.nglob, mesh.ndir, setup="device", **kw)
    rng = np.random.default_rng(1)
    for group in ("dense", "W", "V"):
        for dh, dd in zip(getattr(host, group), getattr(dev, group)):
            x = rng.uniform(-1, 1, dh.in_size)
            assert rel_l2(dd(x), dh(x)) < 1e-11, group
    xh, rh = host.solve(b, x0, tol=1e-12)
    xd, rd = dev.solve(b, x0, tol=1e-12)
    assert rd.converged and rel_l2(xd, xh) < 1e-10
    assert abs(rd.iterations - rh.iterations) <= 2


def test_device_condensation_rejects_an_indefinite_interior_block():
    import ctypes
    ne, nc = 2, 4
    K = -np.tile(np.eye(nc), (ne, 1, 1))  # negative definite
    import torch
    Kd = torch.tensor(K, device="cuda")
    S = torch.empty((ne, 2, 2), dtype=torch.float64, device="cuda")
    W = torch.empty((ne, 2, 4), dtype=torch.float64, device="cuda")
    V = torch.empty((ne, 4, 4), dtype=torch.float64, device="cuda")
    bm = np.array([0, 3], dtype=np.int32)
    im = np.array([1, 2], dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    rc = nb.lib().nkb_condense(ne, nc, ctypes.c_void_p(Kd.data_ptr()), 2, bm.ctypes.data_as(ip), 2,
                               im.ctypes.data_as(ip), None, ctypes.c_void_p(S.data_ptr()),
                               ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(V.data_ptr()), 0,
                               None)
    assert rc == nb.C.NKB_ERR_INVALID
    assert b"positive definite" in nb.lib().nkb_last_error()
