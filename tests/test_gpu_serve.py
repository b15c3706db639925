"""Serving loop on the device: a mixed stream of FP64 and mixed-precision
requests on several meshes, served concurrently, gives for every request
exactly the bits it gets when served alone, and solves the system that
operators built with the request's lambda define."""
import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200.serve import CudaBackend, Request, Scheduler, rhs_for, summarize
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _stream():
    rng = np.random.default_rng(42)
    reqs = []
    for i in range(12):
        n, P = [(3, 3), (4, 2), (3, 4)][i % 3]
        mixed = bool(i % 2)
        reqs.append(Request(i, 0.002 * i, n, P, float(rng.uniform(0.1, 10.0)),
                            1e-8 if mixed else 1e-10, mixed, int(rng.integers(1 << 30))))
    return reqs


def test_served_in_mix_equals_served_alone():
    reqs = _stream()
    sch = Scheduler(CudaBackend(), 4 << 30, max_active=6, keep_x=True)
    mix = sch.run(reqs)
    sch.close()
    s = summarize(mix, reqs)
    assert s["converged"] == len(reqs)
    for k in (0, 1, 5, 10):
        alone = Scheduler(CudaBackend(), 4 << 30, max_active=1, keep_x=True)
        r = alone.run([reqs[k]])[0]
        alone.close()
        assert r.iterations == mix[k].iterations
        assert np.array_equal(r.x, mix[k].x), k


def test_served_solution_matches_direct_solve():
    reqs = _stream()[:2]   # one FP64 (tol 1e-10), one mixed (tol 1e-8)
    sch = Scheduler(CudaBackend(), 4 << 30, keep_x=True)
    res = sch.run(reqs)
    sch.close()
    for req, r in zip(reqs, res):
        m = nb.BoxMesh("hex", req.n, req.P + 1, req.P + 2, amp=0.05)
        gmap, nglob, ndir = m.assembly()
        op = nb.Operator("helmholtz", m)
        op.set_factors(req.lam)
        S = nb.GlobalLinSys([op], gmap, nglob, ndir)
        x, rep = S.solve(rhs_for(req, m.nelmt * m.nc), tol=1e-12)
        assert r.converged
        # |x - x*| / |x*| <= cond(A) |r| / |b|, with cond(A) ~ 1e2 on these meshes
        assert rel_l2(r.x, x) < (1e-4 if req.mixed else 1e-6)
