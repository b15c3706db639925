"""Non-blocking solves, clones and per-system lambda on the device: the
machinery the serving loop drives. A solve advanced by polls must give the
same bits as the blocking solve, concurrent clones must not disturb each
other, and a clone's own lambda must solve the same system as operators built
with that lambda."""
import numpy as np
import pytest

import nektar_b200 as nb
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _system(n, nm, lam=1.0, mixed=False):
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05, coords=True)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(lam)
    ops32 = None
    if mixed:
        op32 = nb.Operator("helmholtz", m, precision="fp32")
        op32.set_factors(lam)
        ops32 = [op32]
    S = nb.GlobalLinSys([op], gmap, nglob, ndir, ops32=ops32)
    return m, S, (op, ops32)


def _device(arr):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).cuda()


def _solve_polled(S, b, tol, mixed=False):
    torch = _torch()
    bd = _device(b)
    xd = torch.zeros_like(bd)
    torch.cuda.synchronize()  # the system's own stream does not wait for torch's
    S.begin(bd.data_ptr(), xd.data_ptr(), tol=tol, check_interval=8, mixed=mixed)
    polls = 0
    while not S.poll():
        polls += 1
    rep = S.end()
    torch.cuda.synchronize()
    return xd.cpu().numpy(), rep, polls


@pytest.mark.parametrize("mixed", [False, True])
def test_polled_solve_is_bitwise_the_blocking_solve(mixed):
    m, S, keep = _system(4, 5, mixed=mixed)
    b = np.random.default_rng(3).uniform(-1, 1, m.nelmt * m.nc)
    torch = _torch()
    bd = _device(b)
    xd = torch.zeros_like(bd)
    torch.cuda.synchronize()
    rep0 = S.solve_device(bd.data_ptr(), xd.data_ptr(), tol=1e-11, check_interval=8,
                          mixed=mixed)
    torch.cuda.synchronize()
    x0 = xd.cpu().numpy()
    x1, rep1, polls = _solve_polled(S, b, 1e-11, mixed)
    assert rep0.converged and rep1.converged
    assert rep0.iterations == rep1.iterations
    assert np.array_equal(x0, x1)
    assert polls >= 1


def test_concurrent_clones_match_solo_solves():
    """Two clones of one system solved with interleaved polls on their own
    streams give exactly what each gives alone."""
    torch = _torch()
    m, S, keep = _system(4, 5)
    C = S.clone()
    rng = np.random.default_rng(7)
    b1 = rng.uniform(-1, 1, m.nelmt * m.nc)
    b2 = rng.uniform(-1, 1, m.nelmt * m.nc)
    solo1, _, _ = _solve_polled(S, b1, 1e-10)
    solo2, _, _ = _solve_polled(C, b2, 1e-10)
    d1, d2 = _device(b1), _device(b2)
    x1, x2 = torch.zeros_like(d1), torch.zeros_like(d2)
    torch.cuda.synchronize()
    S.begin(d1.data_ptr(), x1.data_ptr(), tol=1e-10, check_interval=8)
    C.begin(d2.data_ptr(), x2.data_ptr(), tol=1e-10, check_interval=8)
    done = [False, False]
    while not all(done):
        if not done[0]:
            done[0] = S.poll()
        if not done[1]:
            done[1] = C.poll()
    r1, r2 = S.end(), C.end()
    torch.cuda.synchronize()
    assert r1.converged and r2.converged
    assert np.array_equal(x1.cpu().numpy(), solo1)
    assert np.array_equal(x2.cpu().numpy(), solo2)
    sh, inst = S.footprint()
    sh2, inst2 = C.footprint()
    assert sh == sh2 and sh > 0 and inst > 0 and inst2 > 0
    C.close()


@pytest.mark.parametrize("lam", [0.1, 7.5])
def test_set_lambda_matches_operators_built_with_lambda(lam):
    m, S, keep = _system(3, 5, lam=1.0)
    m2, S2, keep2 = _system(3, 5, lam=lam)
    C = S.clone()
    C.set_lambda(lam)
    assert rel_l2(C.diag_inv(), S2.diag_inv()) < 1e-13
    b = np.random.default_rng(11).uniform(-1, 1, m.nelmt * m.nc)
    xc, rc = C.solve(b, tol=1e-12)
    x2, r2 = S2.solve(b, tol=1e-12)
    assert rc.converged and r2.converged
    assert abs(rc.iterations - r2.iterations) <= 3
    assert rel_l2(xc, x2) < 1e-10
    # the parent keeps its own lambda
    x1, _ = S.solve(b, tol=1e-12)
    assert rel_l2(x1, x2) > 1e-6
    C.close()


def test_poll_and_end_without_a_solve_are_errors():
    m, S, keep = _system(2, 3)
    with pytest.raises(nb.NektarB200Error) as e:
        S.poll()
    assert e.value.code == nb.C.NKB_ERR_INVALID
    with pytest.raises(nb.NektarB200Error) as e:
        S.end()
    assert e.value.code == nb.C.NKB_ERR_INVALID
