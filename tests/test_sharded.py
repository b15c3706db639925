"""The sharded solve on the CPU: two gloo ranks, each with its slab of
elements, the oracle's element operator, interface sums and dot products
over the process group; the result equals the one-rank solve and the dense
solution."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nektar_b200.sharded import ShardedSystem, partition


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(n=3, nm=5):
    import nektar_b200 as nb
    from oracle import oracle as O
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    T = dict(m.T)
    T["w"] = m.T["ws"]
    nt, nc = m.nt, m.nc

    def apply_range(lo, hi):
        jac = m.jac[lo * nt:hi * nt]
        df = np.ascontiguousarray(m.df[:, lo * nt:hi * nt])
        return lambda x: O.helmholtz("hex", nm, m.nq, hi - lo, T, jac, df, x, 1.0, True)

    def diag_range(lo, hi):
        jac = m.jac[lo * nt:hi * nt]
        df = np.ascontiguousarray(m.df[:, lo * nt:hi * nt])
        return O.helmholtz_diag("hex", nm, m.nq, hi - lo, T, jac, df, 1.0, True)

    rng = np.random.default_rng(4)
    b = rng.uniform(-1, 1, m.nelmt * nc)
    xd = rng.uniform(-1, 1, ndir)  # Dirichlet values, consistent
    x0 = np.where(gmap < ndir, xd[np.minimum(gmap, ndir - 1)], 0.0)
    return m, gmap, nglob, ndir, apply_range, diag_range, b, x0


def _solve(world, rank, pg, out):
    m, gmap, nglob, ndir, apply_range, diag_range, b, x0 = _problem()
    lo, hi = partition(m.nelmt, world, rank)
    nc = m.nc
    S = ShardedSystem(gmap, None, nc, ndir, lo, hi, apply_range(lo, hi), diag_range(lo, hi), pg)
    x, it = S.solve(b[lo * nc:hi * nc], x0[lo * nc:hi * nc], tol=1e-12)
    out[rank] = (lo, hi, x, it)


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        _solve(world, rank, dist, out)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_partition_covers_every_element_once():
    for n, w in ((10, 3), (7, 7), (5, 2)):
        ranges = [partition(n, w, r) for r in range(w)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))


def test_one_rank_solve_matches_dense_solution():
    m, gmap, nglob, ndir, apply_range, diag_range, b, x0 = _problem()
    out = {}
    _solve(1, 0, None, out)
    _, _, x, it = out[0]
    # dense reference: element matrices from the operator
    nc, ne = m.nc, m.nelmt
    A = apply_range(0, ne)
    G = np.zeros((nglob, nglob))
    for j in range(nc):
        e = np.zeros(ne * nc)
        e[j::nc] = 1.0
        col = A(e).reshape(ne, nc)
        for el in range(ne):
            G[gmap[el * nc:(el + 1) * nc], gmap[el * nc + j]] += col[el]
    bg = np.zeros(nglob)
    np.add.at(bg, gmap, b)
    xd = np.zeros(nglob)
    for l, g_ in enumerate(gmap):
        if g_ < ndir:
            xd[g_] = x0[l]
    rhs = bg - G @ xd
    xg = xd.copy()
    xg[ndir:] = np.linalg.solve(G[ndir:, ndir:], rhs[ndir:])
    assert np.abs(x - xg[gmap]).max() < 1e-9 * np.abs(xg).max()
    assert it > 10


def test_two_gloo_ranks_match_one_rank():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    one = {}
    _solve(1, 0, None, one)
    x1, it1 = one[0][2], one[0][3]
    nc = 5 ** 3
    for r in range(world):
        lo, hi, x, it = res[r]
        assert np.abs(x - x1[lo * nc:hi * nc]).max() < 1e-10 * np.abs(x1).max()
        assert abs(it - it1) <= max(5, it1 // 20)  # sums in another order near tol 1e-12
