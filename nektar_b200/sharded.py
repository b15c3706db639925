"""A Helmholtz solve sharded over ranks by element partition: the parallel
form of GlobalLinSysIterativeFull + NekLinSysIterCG that MPI runs of the
reference use (one partition per rank, MeshPartition.cpp:99; the shared
dofs summed across partitions by AssemblyMapCG::UniversalAssemble,
AssemblyMapCG.cpp:2894-2906; the three dot products of an iteration summed
in one all-reduce, NekLinSysIterCG.cpp:310).

Every rank holds a contiguous block of elements (its partition) and numbers
the global dofs they touch

    [Dirichlet | free, this rank only | free shared, owned | free shared, others']

A dof touched by several ranks is owned by the lowest of them, which alone
counts it in dot products. `shard_plans` builds, from the whole mesh's
local -> global map, every rank's numbering and its exchange plan: the dofs
it shares with each neighbour rank (in increasing mesh-wide id, the order
both sides use) and, per shared dof, where each sharing rank's value lands,
in rank order. Summing in rank order gives every rank the same bits.

Two solvers use the plans:

* `DeviceShardGroup` -- the device CG (`nkb_shard_group_*`): every vector on
  the GPU; the exchange by NCCL send/recv with each neighbour and the dot
  sums by one NCCL all-reduce (one shard per process and GPU, `make_comm`),
  or, with all shards in one process on one GPU, by device copies (the
  sharded recurrence run on one GPU).
* `ShardedSystem` -- the same recurrence on the host, one rank per process
  of a torch.distributed group (gloo: host tensors; nccl: device tensors),
  the exchange by point-to-point sends to the neighbours. It is the host
  restatement the device group is checked against, and it takes any element
  operator (`apply`), e.g. the oracle's.
"""
import ctypes

import numpy as np


def partition(nelmt, world, rank):
    """Contiguous element range [lo, hi) of a rank (MeshPartition's blocks
    of a box mesh numbered layer by layer are such slabs)."""
    base, extra = divmod(nelmt, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_plans(gmap, ndir, world, elem_off=None, nc=None):
    """Every rank's numbering and exchange plan (a list of dicts, one per
    rank). gmap: the whole mesh's local -> global map (element-major);
    elem_off: element offsets into it (nelmt + 1), or nc for equal elements.

    Per rank: lo, hi (its elements); gid (its dofs' mesh-wide ids in its
    numbering); lmap (its elements' local -> its numbering); nglob, ndir,
    nint, nown; dir_owned (uint8 over its Dirichlet dofs); shared, sptr,
    ssrc (per shared dof the sources in rank order: -1 its own value, else
    a position in its receive buffer); nbr, nptr, nidx (per neighbour the
    dofs sent, in increasing mesh-wide id)."""
    gmap = np.asarray(gmap, dtype=np.int64)
    if elem_off is None:
        elem_off = np.arange(gmap.size // nc + 1, dtype=np.int64) * nc
    elem_off = np.asarray(elem_off, dtype=np.int64)
    nelmt = elem_off.size - 1
    nglob = int(gmap.max()) + 1
    ranges = [partition(nelmt, world, r) for r in range(world)]
    touched = [np.unique(gmap[elem_off[lo]:elem_off[hi]]) for lo, hi in ranges]
    count = np.zeros(nglob, dtype=np.int64)
    first = np.full(nglob, world, dtype=np.int64)
    for r, t in enumerate(touched):
        count[t] += 1
        first[t] = np.minimum(first[t], r)
    # (gid, rank) of every shared dof, sorted by gid then rank
    pg = np.concatenate([t[count[t] > 1] for t in touched])
    pr = np.concatenate([np.full(int((count[t] > 1).sum()), r) for r, t in enumerate(touched)])
    o = np.lexsort((pr, pg))
    pg, pr = pg[o], pr[o]
    plans = []
    for r, ((lo, hi), t) in enumerate(zip(ranges, touched)):
        dirm = t < ndir
        sh = count[t] > 1
        D = t[dirm]
        Fi = t[~dirm & ~sh]
        Fo = t[~dirm & sh & (first[t] == r)]
        Fx = t[~dirm & sh & (first[t] != r)]
        gid = np.concatenate([D, Fi, Fo, Fx])
        pos = np.full(nglob, -1, dtype=np.int64)
        pos[gid] = np.arange(gid.size)
        lmap = pos[gmap[elem_off[lo]:elem_off[hi]]]
        # neighbours and the dofs shared with each
        mine = np.zeros(nglob, dtype=bool)
        mine[t[sh]] = True
        sel = mine[pg]
        g_r, q_r = pg[sel], pr[sel]
        nbr = np.unique(q_r[q_r != r])
        common = [np.sort(g_r[q_r == q]) for q in nbr]
        nptr = np.zeros(nbr.size + 1, dtype=np.int64)
        nptr[1:] = np.cumsum([c.size for c in common])
        nidx = (np.concatenate([pos[c] for c in common]) if nbr.size
                else np.zeros(0, dtype=np.int64))
        # sources of every shared dof in rank order
        src = np.full(g_r.size, -1, dtype=np.int64)
        for k, (q, c) in enumerate(zip(nbr, common)):
            m = q_r == q
            src[m] = nptr[k] + np.searchsorted(c, g_r[m])
        ug, start = np.unique(g_r, return_index=True)
        sptr = np.append(start, g_r.size)
        plans.append(dict(
            rank=r, lo=lo, hi=hi, gid=gid, lmap=lmap.astype(np.int32), nglob=int(gid.size),
            ndir=int(D.size), nint=int(Fi.size), nown=int(Fi.size + Fo.size),
            dir_owned=(first[D] == r).astype(np.uint8), shared=pos[ug].astype(np.int32),
            sptr=sptr.astype(np.int32), ssrc=src.astype(np.int32), nbr=nbr.astype(np.int32),
            nptr=nptr.astype(np.int32), nidx=nidx.astype(np.int32)))
    return plans


def unpack(plan, v, recv):
    """Each shared dof of v (this rank's numbering) = the sum of the sharing
    ranks' values in rank order (what k_unpack does)."""
    out = v.copy()
    sp, src, g = plan["sptr"].astype(np.int64), plan["ssrc"], plan["shared"]
    if not g.size:
        return out
    n = np.diff(sp)
    acc = np.zeros(g.size)
    for j in range(int(n.max())):  # j-th source of every shared dof, in rank order
        m = n > j
        c = src[sp[:-1][m] + j]
        acc[m] += np.where(c < 0, v[g[m]], recv[np.maximum(c, 0)])
    out[g] = acc
    return out


class ShardedSystem:
    """One rank's part of the sharded solve on the host.

    gmap, sign: the whole mesh's local -> global map (nelmt * nc entries,
    element-major, Dirichlet dofs numbered first); nc local modes per
    element; lo, hi the rank's elements (partition(nelmt, world, rank));
    apply(x_loc) -> y_loc the rank's element operator on its local vector;
    diag_loc the rank's element diagonals (for Jacobi); pg the
    torch.distributed module or None for one rank."""

    def __init__(self, gmap, sign, nc, ndir, lo, hi, apply, diag_loc, pg=None):
        import torch
        self.torch, self.pg = torch, pg
        world = 1 if pg is None else pg.get_world_size()
        rank = 0 if pg is None else pg.get_rank()
        p = shard_plans(gmap, ndir, world, nc=nc)[rank]
        if (p["lo"], p["hi"]) != (lo, hi):
            raise ValueError("elements [%d,%d) are not rank %d's partition" % (lo, hi, rank))
        self.plan, self.apply = p, apply
        self.lmap = p["lmap"].astype(np.int64)
        sg = np.ones(len(gmap)) if sign is None else np.asarray(sign, np.float64)
        self.sign_r = sg[lo * nc:hi * nc]
        self.nd, self.nint, self.nown = p["ndir"], p["nint"], p["nown"]
        self.n = p["nglob"]
        self.diag = self._assemble(np.asarray(diag_loc, np.float64), absolute=True)
        self.dinv = np.zeros(self.n)
        self.dinv[self.nd:] = 1.0 / self.diag[self.nd:]

    # -- communication -------------------------------------------------------
    def _exchange(self, v):
        """v summed over the ranks at the shared dofs: the values each
        neighbour shares sent to it, its values received, rank-order sums."""
        p = self.plan
        if self.pg is None or not p["nbr"].size:
            return v
        send = np.ascontiguousarray(v[p["nidx"]])
        recv = np.zeros(send.size)
        t = self.torch
        dev = None
        if self.pg.get_backend() == "nccl":  # NCCL moves device tensors only
            dev = "cuda:%d" % t.cuda.current_device()
        ts = t.from_numpy(send) if dev is None else t.from_numpy(send).to(dev)
        tr = t.zeros(recv.size, dtype=t.float64, device=dev or "cpu")
        reqs = []
        for k, q in enumerate(p["nbr"]):
            a, b = int(p["nptr"][k]), int(p["nptr"][k + 1])
            reqs.append(self.pg.isend(ts[a:b], int(q)))
            reqs.append(self.pg.irecv(tr[a:b], int(q)))
        for rq in reqs:
            rq.wait()
        recv = tr.cpu().numpy()
        return unpack(p, v, recv)

    def _allreduce(self, arr):
        if self.pg is None:
            return arr
        t = self.torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64))
        if self.pg.get_backend() == "nccl":
            d = t.to("cuda:%d" % self.torch.cuda.current_device())
            self.pg.all_reduce(d)
            return d.cpu().numpy()
        self.pg.all_reduce(t)
        return t.numpy()

    def _assemble(self, y_loc, absolute=False):
        """Rank-local assemble, then the shared dofs summed over ranks."""
        s = self.sign_r * self.sign_r if absolute else self.sign_r
        out = np.zeros(self.n)
        np.add.at(out, self.lmap, s * y_loc)
        return self._exchange(out)

    def _matvec(self, x):
        return self._assemble(self.apply(self.sign_r * x[self.lmap]))

    def _dots(self, *pairs):
        """Dot products over the rank's own free dofs (and for |b|^2 its own
        Dirichlet ones), summed over the ranks."""
        f = slice(self.nd, self.nd + self.nown)
        return self._allreduce(np.array([np.sum(a[f] * b[f]) for a, b in pairs]))

    # -- solve ---------------------------------------------------------------
    def solve(self, b_loc, x0_loc, tol=1e-10, maxit=5000):
        """Rank's local rhs and local Dirichlet values -> rank's local
        solution, iterations. The recurrence and the stopping rule of
        NekLinSysIterCG::DoConjugateGradient (reduced communication)."""
        x0_loc = np.asarray(x0_loc, np.float64)
        bg = self._assemble(np.asarray(b_loc, np.float64) - self.apply(x0_loc))
        own_d = self.plan["dir_owned"].astype(bool)
        bdir = self._allreduce(np.array([np.sum(bg[:self.nd][own_d] ** 2)]))[0]
        r = bg.copy()
        r[:self.nd] = 0.0
        bnorm, eps = self._dots((r, r), (r, r))
        bnorm += bdir
        bnorm = bnorm if bnorm > 1e-6 else 1.0
        x = np.zeros(self.n)
        it = 0
        if eps >= tol * tol * bnorm:
            w = self.dinv * r
            s = self._matvec(w)
            s[:self.nd] = 0.0
            rho, mu = self._dots((r, w), (s, w))
            p, q = w.copy(), s.copy()
            alpha, beta, it = rho / mu, 0.0, 1
            while True:
                x += alpha * p
                r -= alpha * q
                w = self.dinv * r
                s = self._matvec(w)
                s[:self.nd] = 0.0
                rho_new, mu, eps = self._dots((r, w), (s, w), (r, r))
                if eps < tol * tol * bnorm or it >= maxit:
                    break
                beta = rho_new / rho
                alpha = rho_new / (mu - rho_new * beta / alpha)
                rho = rho_new
                p = w + beta * p
                q = s + beta * q
                it += 1
        return x0_loc + self.sign_r * x[self.lmap], it


def device_apply(op_factory, lo, hi):
    """apply() over a rank's elements [lo, hi) with device operators built by
    op_factory(lo, hi) (a Helmholtz Operator of those elements)."""
    op = op_factory(lo, hi)
    return lambda x: op(x)


def make_comm(pg, device):
    """The NCCL communicator of the device group over a torch.distributed
    group (any backend): rank 0's unique id broadcast to every rank; with pg
    None a communicator of one rank. Returns an nkb_comm handle (close with
    close_comm).

    torch is imported first: the library binds the libnccl.so.2 the process
    has loaded, and torch brings its own; were the system's bound first, a
    later `import torch` would find that older copy under the same name."""
    import torch  # noqa: F401

    from nektar_b200 import check, lib
    world = 1 if pg is None else pg.get_world_size()
    rank = 0 if pg is None else pg.get_rank()
    idb = (ctypes.c_ubyte * 128)()
    if rank == 0:
        check(lib().nkb_comm_unique_id(idb))
    if pg is not None:
        box = [bytes(idb)]
        pg.broadcast_object_list(box, src=0)
        idb = (ctypes.c_ubyte * 128).from_buffer_copy(box[0])
    h = ctypes.c_void_p()
    check(lib().nkb_comm_create(idb, world, rank, device, ctypes.byref(h)))
    return h


def close_comm(h):
    from nektar_b200 import lib
    if h:
        lib().nkb_comm_destroy(h)


class DeviceShardGroup:
    """The device CG over shards (nkb_shard_group_*).

    plans: the plans (shard_plans) of the shards this process holds; ops:
    per held shard, its FP64 Helmholtz operators (collections of its
    elements, in local order); comm: an NCCL communicator (make_comm) when
    this process holds one shard of a multi-GPU solve, else None (every
    shard in this process, on `device`). sign: per held shard its local
    signs, or None."""

    def __init__(self, plans, ops, comm=None, device=0, signs=None):
        import nektar_b200 as nb
        from nektar_b200 import _capi as C
        self.plans = list(plans)
        self.systems = []
        for k, (p, o) in enumerate(zip(self.plans, ops)):
            sg = None if signs is None else signs[k]
            self.systems.append(nb.GlobalLinSys(o, p["lmap"], p["nglob"], p["ndir"], sign=sg,
                                                device=device))
        self._keep = []
        cp = (C.ShardPlan * len(self.plans))()

        def arr(a, ctype):
            a = np.ascontiguousarray(a, dtype=ctype)
            self._keep.append(a)
            return a

        for k, p in enumerate(self.plans):
            c = cp[k]
            c.rank, c.nint, c.nown = p["rank"], p["nint"], p["nown"]
            c.dir_owned = arr(p["dir_owned"], np.uint8).ctypes.data_as(
                ctypes.POINTER(ctypes.c_ubyte))
            c.nshared = int(p["shared"].size)
            c.shared = arr(p["shared"], np.int32).ctypes.data_as(C.ip)
            c.sptr = arr(p["sptr"], np.int32).ctypes.data_as(C.ip)
            c.ssrc = arr(p["ssrc"], np.int32).ctypes.data_as(C.ip)
            c.nnbr = int(p["nbr"].size)
            c.nbr = arr(p["nbr"], np.int32).ctypes.data_as(C.ip)
            c.nptr = arr(p["nptr"], np.int32).ctypes.data_as(C.ip)
            c.nidx = arr(p["nidx"], np.int32).ctypes.data_as(C.ip)
        hs = (ctypes.c_void_p * len(self.systems))(*[s.h.value for s in self.systems])
        g = ctypes.c_void_p()
        nb.check(nb.lib().nkb_shard_group_create(hs, cp, len(self.systems), comm,
                                                 ctypes.byref(g)))
        self.h = g
        self._cp = cp

    def solve(self, b_locs, x_locs=None, tol=1e-9, maxit=5000, check_interval=16,
              use_graph=True):
        """Host arrays per held shard: local rhs and local Dirichlet values
        -> local solutions, reports."""
        import nektar_b200 as nb
        from nektar_b200 import _capi as C
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in b_locs]
        xs = [np.zeros(b.size) if x_locs is None else
              np.ascontiguousarray(x, dtype=np.float64).copy()
              for b, x in zip(bs, x_locs if x_locs is not None else [None] * len(bs))]
        bp = (ctypes.c_void_p * len(bs))(*[b.ctypes.data for b in bs])
        xp = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        reps = (C.CGReport * len(bs))()
        opts = nb.GlobalLinSys._opts(tol, maxit, check_interval, use_graph)
        nb.check(nb.lib().nkb_shard_group_solve(self.h, bp, xp, ctypes.byref(opts), reps,
                                                nb.HOST_PTRS))
        return xs, list(reps)

    def close(self):
        import nektar_b200 as nb
        if getattr(self, "h", None):
            nb.lib().nkb_shard_group_destroy(self.h)
            self.h = None
        for s in getattr(self, "systems", []):
            s.close()
        self.systems = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
