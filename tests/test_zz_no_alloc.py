"""nkb_op_apply_host_static: the host-pointer operator apply that allocates no
device memory (for callers that must stay inside a device-memory budget fixed
at start-up, or must not take the synchronisation an allocation can cause).
It stages through one static 32 MiB device array instead of cudaMalloc'd
buffers. Checked through the C ABI against nkb_op_apply with host pointers on
two calls in a row (the array keeps the previous call's contents). Collected
last so that a run stopping at the first failure has run every other test."""

import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200 import _capi as C
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _apply_existing(op, x):
    nouts = 3 if op.optype == nb.PHYSDERIV else 1
    outs = [np.zeros(op.out_size) for _ in range(nouts)] + [None] * (3 - nouts)
    nb.check(C.lib().nkb_op_apply(op.h, x.ctypes.data,
                                  *[None if o is None else o.ctypes.data for o in outs],
                                  C.HOST_PTRS, None))
    return outs[:nouts]


def _apply_static(op, x):
    nouts = 3 if op.optype == nb.PHYSDERIV else 1
    outs = [np.full(op.out_size, np.nan) for _ in range(nouts)] + [None] * (3 - nouts)
    nb.check(C.lib().nkb_op_apply_host_static(
        op.h, x.ctypes.data, *[None if o is None else o.ctypes.data for o in outs], None))
    return outs[:nouts]


@pytest.mark.parametrize("shape,optype,nm", [("hex", "helmholtz", 7), ("tet", "physderiv", 5),
                                             ("prism", "iproduct", 4)])
def test_static_apply_matches_allocating_apply(shape, optype, nm):
    m = nb.BoxMesh(shape, 3, nm, nm + 1, amp=0.05)
    op = nb.Operator(optype, m)
    rng = np.random.default_rng(nm)
    for call in range(2):  # two calls in a row: the shared array keeps old data
        x = rng.uniform(-1, 1, op.in_size)
        ref = _apply_existing(op, x)
        got = _apply_static(op, x)
        for g, r in zip(got, ref):
            assert np.all(np.isfinite(g))
            assert rel_l2(g, r) < TOL64, (call, rel_l2(g, r))


def test_static_apply_allocates_no_device_memory():
    """On a freshly created operator whose staging would take about 32 MB, the
    static apply leaves the device's free memory where it was (an allocating
    apply would take it). A first call on another operator loads the library's
    device code, so lazy module loading cannot count against the call."""
    import torch
    small = nb.Operator("helmholtz", nb.BoxMesh("hex", 2, 4, 5, amp=0.05))
    _apply_static(small, np.ones(small.in_size))
    m = nb.BoxMesh("hex", 18, 7, 8, amp=0.05)  # in + out = 4,000,752 doubles
    op = nb.Operator("helmholtz", m)
    x = np.random.default_rng(9).uniform(-1, 1, op.in_size)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got = _apply_static(op, x)[0]
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (4 << 20), (free0, free1)
    assert rel_l2(got, _apply_existing(op, x)[0]) < TOL64


def test_static_apply_rejects_operators_beyond_the_limit():
    # 19^3 P=6 Hex Helmholtz: 2 x 6859 x 343 doubles > 4 Mi doubles
    m = nb.BoxMesh("hex", 19, 7, 8, amp=0.05)
    op = nb.Operator("helmholtz", m)
    x = np.zeros(op.in_size)
    y = np.zeros(op.out_size)
    rc = C.lib().nkb_op_apply_host_static(op.h, x.ctypes.data, y.ctypes.data, None, None, None)
    assert rc == C.NKB_ERR_INVALID
    assert b"static area" in C.lib().nkb_last_error()
