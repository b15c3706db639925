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


def _box(n=3, nm=5):
    import nektar_b200 as nb
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    return m, np.asarray(gmap), nglob, ndir


@pytest.mark.parametrize("world", [1, 2, 3, 4, 5, 7])
def test_shard_plans_number_own_and_pair_every_dof(world):
    """Each rank's numbering covers the dofs its elements touch (Dirichlet,
    then its own free dofs, then the shared free dofs it owns, then the
    others'); every dof is owned once; two neighbours list the same shared
    dofs in the same order; a shared dof has one source per sharing rank,
    its own value once. 27 elements over 4, 5 or 7 ranks give partitions that
    end mid-layer."""
    from nektar_b200.sharded import shard_plans
    m, gmap, nglob, ndir = _box()
    nc = m.nc
    plans = shard_plans(gmap, ndir, world, nc=nc)
    owners = np.zeros(nglob, dtype=np.int64)
    touch = np.zeros(nglob, dtype=np.int64)
    for p in plans:
        gid, nd, nint, nown = p["gid"], p["ndir"], p["nint"], p["nown"]
        assert np.array_equal(gid[p["lmap"]], gmap[p["lo"] * nc:p["hi"] * nc])
        assert np.unique(gid).size == gid.size
        assert (gid[:nd] < ndir).all() and (gid[nd:] >= ndir).all()
        touch[gid] += 1
        owners[gid[nd:nd + nown]] += 1
        owners[gid[:nd][p["dir_owned"].astype(bool)]] += 1
    assert (owners == 1).all()
    for p in plans:
        gid, nd, nint = p["gid"], p["ndir"], p["nint"]
        assert (touch[gid[nd:nd + nint]] == 1).all()
        assert (touch[gid[nd + nint:]] > 1).all()
        sh = p["shared"]
        assert set(sh.tolist()) == set(np.flatnonzero(touch[gid] > 1).tolist())
        nsrc = np.diff(p["sptr"])
        assert np.array_equal(nsrc, touch[gid[sh]])
        for k in range(sh.size):
            src = p["ssrc"][p["sptr"][k]:p["sptr"][k + 1]]
            assert (src == -1).sum() == 1
        for k, q in enumerate(p["nbr"]):
            pq = plans[q]
            kk = list(pq["nbr"]).index(p["rank"])
            mine = gid[p["nidx"][p["nptr"][k]:p["nptr"][k + 1]]]
            theirs = pq["gid"][pq["nidx"][pq["nptr"][kk]:pq["nptr"][kk + 1]]]
            assert np.array_equal(mine, theirs) and (np.diff(mine) > 0).all()


@pytest.mark.parametrize("world", [2, 3, 5])
def test_plan_exchange_gives_every_rank_the_assembled_vector(world):
    """Rank-local assembles of a local vector, exchanged through the plans
    (each rank's send slice into its neighbours' receive slices) and summed
    in rank order, equal the whole mesh's assembled vector at every rank's
    dofs, and carry the same bits on every rank that shares a dof."""
    from nektar_b200.sharded import shard_plans, unpack
    m, gmap, nglob, ndir = _box()
    nc = m.nc
    y = np.random.default_rng(world).uniform(-1, 1, gmap.size)
    full = np.zeros(nglob)
    np.add.at(full, gmap, y)
    plans = shard_plans(gmap, ndir, world, nc=nc)
    part, send = [], []
    for p in plans:
        v = np.zeros(p["nglob"])
        np.add.at(v, p["lmap"].astype(np.int64), y[p["lo"] * nc:p["hi"] * nc])
        part.append(v)
        send.append(v[p["nidx"]])
    done = []
    for p, v in zip(plans, part):
        recv = np.zeros(send[p["rank"]].size)
        for k, q in enumerate(p["nbr"]):
            pq = plans[q]
            kk = list(pq["nbr"]).index(p["rank"])
            recv[p["nptr"][k]:p["nptr"][k + 1]] = send[q][pq["nptr"][kk]:pq["nptr"][kk + 1]]
        out = unpack(p, v, recv)
        assert np.allclose(out, full[p["gid"]], rtol=1e-14, atol=1e-14)
        done.append(out)
    val = {}
    for p, out in zip(plans, done):
        for g, x in zip(p["gid"], out):
            assert val.setdefault(int(g), x) == x
