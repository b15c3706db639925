"""The tcgen05 tensor-core Hex Helmholtz kernel (FP32 operators, TF32 high/low
operands, FP32 accumulation) against the FP64 oracle at the FP32 bar
(relative L2 <= 2e-5), in the mixed-precision CG, and the device error word
of bounded waits read back by the host."""
import numpy as np
import pytest

import nektar_b200 as nb
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL32 = 2e-5


def _oracle_T(m):
    T = dict(m.T)
    T["w"] = m.T["ws"]
    return T


def _tc_op(monkeypatch, m, lam):
    monkeypatch.setenv("NKB_HEX_VARIANT", "5")
    op = nb.Operator("helmholtz", m, precision="fp32")
    monkeypatch.delenv("NKB_HEX_VARIANT")
    assert "tcgen05" in op.kernel(), op.kernel()
    op.set_factors(lam)
    return op


def _apply32(op, x):
    import torch
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.empty(op.out_size, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    op.apply_device(xd.data_ptr(), yd.data_ptr(), stream=s.cuda_stream)
    s.synchronize()
    op.check_error()
    return yd.double().cpu().numpy()


def _tf32_trunc(a):
    """What a TF32 MMA reads of an FP32 operand (the top 19 bits)."""
    return (np.asarray(a, dtype=np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


@pytest.mark.parametrize("colw", [0, 1, 2])
@pytest.mark.parametrize("n,ks", [(16, 1), (32, 1), (64, 1), (16, 2), (32, 2)])
def test_tc_building_blocks_compute_a_times_b(colw, n, ks):
    """One 128-row tile through the kernel's operand writers (its row writer,
    its rotated column writer, its padded-layout column writer; TF32
    high/low parts, K-major), K-major
    B table, MMA pair, commit and
    tensor-memory read-back: D = A B to FP32-class accuracy (B is read as
    TF32 by the hardware)."""
    import ctypes
    from nektar_b200 import _capi as C
    rng = np.random.default_rng(17 + n + ks + colw)
    K = 8 * ks
    A = rng.uniform(-1, 1, (128, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, n)).astype(np.float32)
    D = np.zeros((128, n), dtype=np.float32)
    info = (ctypes.c_uint * 2)()
    fp = ctypes.POINTER(ctypes.c_float)
    nb.check(C.lib().nkb_tc_selftest(colw, n, ks, A.ctypes.data_as(fp), B.ctypes.data_as(fp),
                                     D.ctypes.data_as(fp), info))
    assert info[1] == 1, "MMA completion wait did not complete"
    ref = A.astype(np.float64) @ _tf32_trunc(B).astype(np.float64)
    err = np.abs(D - ref).max() / np.abs(ref).max()
    assert err < 1e-5, (err, D[:2, :4], ref[:2, :4], info[0])


# element counts chosen to leave the last tile partly filled (2 elements per
# tile at nq 6-8, 1 at nq 9-10, up to 10 at nq 3)
@pytest.mark.parametrize("n,nm", [(3, 2), (2, 3), (3, 4), (3, 5), (3, 6), (3, 7), (2, 8), (2, 9),
                                  (1, 7)])
@pytest.mark.parametrize("amp", [0.05, 0.0])
def test_tc_hex_helmholtz_matches_oracle(monkeypatch, n, nm, amp):
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=amp)
    x = np.random.default_rng(nm).uniform(-1, 1, m.nelmt * m.nc)
    yo = O.helmholtz("hex", nm, m.nq, m.nelmt, _oracle_T(m), m.jac, m.df, x, 1.7, m.deformed)
    op = _tc_op(monkeypatch, m, 1.7)
    assert rel_l2(_apply32(op, x), yo) < TOL32


def test_tc_hex_helmholtz_is_repeatable(monkeypatch):
    """Every application gives the same bits: the stages' shared-memory
    operands, the MMA commits and the tensor-memory reads are ordered."""
    m = nb.BoxMesh("hex", 12, 7, 8, amp=0.05)
    x = np.random.default_rng(3).uniform(-1, 1, m.nelmt * m.nc)
    op = _tc_op(monkeypatch, m, 1.0)
    y0 = _apply32(op, x)
    assert all(np.array_equal(_apply32(op, x), y0) for _ in range(40))


@pytest.mark.parametrize("n,nm", [(4, 7), (3, 9)])
def test_tc_hex_in_mixed_cg_matches_fp64(monkeypatch, n, nm):
    """The mixed-precision CG with the tensor-core operator gathered through
    the map reaches the FP64 criterion and the FP64 solution, within the
    iteration bound the FP32 CUDA-core operator is held to when restarts
    occur (random right-hand sides at high order restart both)."""
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    op32 = _tc_op(monkeypatch, m, 1.0)
    monkeypatch.setenv("NKB_HEX_VARIANT", "5")  # the gathered launch too
    S = nb.GlobalLinSys([op], gmap, nglob, ndir, ops32=[op32])
    b = np.random.default_rng(n).uniform(-1, 1, m.nelmt * m.nc)
    x64, r64 = S.solve(b, tol=1e-12)
    xm, rm = S.solve(b, tol=1e-12, mixed=True, inner_tol=0.1)
    assert "tcgen05" in op32.kernel(gather=True)
    assert rm.converged and rm.rel_residual < 1e-12
    assert rel_l2(xm, x64) < 1e-10, rel_l2(xm, x64)
    assert rm.iterations <= 2.2 * r64.iterations + 20, (rm.iterations, r64.iterations)


def test_bounded_wait_that_gives_up_is_reported(monkeypatch):
    """A wait whose first bound runs out (set to zero polls: the geometry copy
    of the TMA-staged kernel is still drained before the CTA exits) leaves its
    elements unwritten; the host apply returns NKB_ERR_TIMEOUT, the error word
    is cleared, and the next apply with the default bound is correct."""
    m = nb.BoxMesh("hex", 3, 4, 5, amp=0.05)
    x = np.random.default_rng(2).uniform(-1, 1, m.nelmt * m.nc)
    monkeypatch.setenv("NKB_HEX_VARIANT", "0")
    op = nb.Operator("helmholtz", m)
    assert "TMA-staged" in op.kernel(), op.kernel()
    op.set_factors(1.0)
    good = op(x)
    op.set_wait_limit(0)
    with pytest.raises(nb.NektarB200Error) as e:
        op(x)
    assert e.value.code == nb.C.NKB_ERR_TIMEOUT
    op.set_wait_limit(-1)
    assert np.array_equal(op(x), good)
    op.check_error()


def test_tc_wait_that_gives_up_is_reported(monkeypatch):
    """The same for the tensor-core kernel's MMA-completion waits: every
    stage still waits for its MMAs before the tensor memory is read or freed,
    no output is written, and check_error reports the timeout once."""
    m = nb.BoxMesh("hex", 3, 7, 8, amp=0.05)
    x = np.random.default_rng(4).uniform(-1, 1, m.nelmt * m.nc)
    op = _tc_op(monkeypatch, m, 1.0)
    good = _apply32(op, x)
    op.set_wait_limit(0)
    with pytest.raises(nb.NektarB200Error) as e:
        _apply32(op, x)
    assert e.value.code == nb.C.NKB_ERR_TIMEOUT
    op.set_wait_limit(-1)
    assert np.array_equal(_apply32(op, x), good)
