"""A Helmholtz solve sharded over ranks by element partition: the parallel
form of GlobalLinSysIterativeFull + NekLinSysIterCG that MPI runs of the
reference use (one partition per rank, MeshPartition.cpp; the shared dofs
summed across partitions by AssemblyMapCG::UniversalAssemble,
AssemblyMapCG.cpp:2894-2906; the three dot products of an iteration summed
in one all-reduce, NekLinSysIterCG.cpp:310).

Every rank holds a contiguous block of elements (its partition), the global
dofs they touch numbered locally, and a mask of the dofs it owns (a dof on
a partition interface is owned by the lowest rank that touches it, so that
every dot product counts it once). One iteration is: the rank's element
operator on its local vector, its local assemble, one all-reduce of the
interface values (a buffer over all interface dofs, zero where a rank does
not touch them), the vector updates, and one all-reduce of the three dot
products. With one rank there is no exchange and the recurrence is the
device CG's.

The element operator is passed in (apply(x_loc) -> y_loc over the rank's
elements): the device Helmholtz operators on a GPU (`device_apply`), any
restatement elsewhere. The collectives go through torch.distributed: with a
gloo group on host tensors; with an NCCL group the exchange buffers are
copied to the rank's current CUDA device for the all-reduce and back (the
vectors of this form stay on the host). Every rank takes the same collective
steps in the same order, in the last iteration too.
"""
import numpy as np


def partition(nelmt, world, rank):
    """Contiguous element range [lo, hi) of a rank (MeshPartition's blocks
    of a box mesh numbered layer by layer are such slabs)."""
    base, extra = divmod(nelmt, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class ShardedSystem:
    """One rank's part of the sharded solve.

    gmap, sign: the whole mesh's local -> global map (nelmt * nc entries,
    element-major, Dirichlet dofs numbered first); nc local modes per
    element; apply(x_loc) -> y_loc the rank's element operator on its local
    vector; diag_loc the rank's element diagonals (for Jacobi); pg the
    torch.distributed module or None for one rank."""

    def __init__(self, gmap, sign, nc, ndir, lo, hi, apply, diag_loc, pg=None):
        import torch
        self.torch, self.pg = torch, pg
        self.nc, self.ndir, self.apply = nc, int(ndir), apply
        gm = np.asarray(gmap).reshape(-1, nc)
        sg = np.ones(gm.shape) if sign is None else np.asarray(sign, np.float64).reshape(-1, nc)
        self.gmap_r = gm[lo:hi].ravel()
        self.sign_r = sg[lo:hi].ravel()
        self.dofs, self.lmap = np.unique(self.gmap_r, return_inverse=True)  # global ids
        self.free = self.dofs >= self.ndir
        # interface dofs: touched by more than one rank
        world = 1 if pg is None else pg.get_world_size()
        rank = 0 if pg is None else pg.get_rank()
        touch = np.zeros(int(gm.max()) + 1, dtype=np.int64)
        first = np.full(touch.size, world, dtype=np.int64)
        for r in range(world):
            a, b = partition(gm.shape[0], world, r)
            d = np.unique(gm[a:b])
            touch[d] += 1
            first[d] = np.minimum(first[d], r)
        shared = np.nonzero(touch > 1)[0]  # interface dofs, sorted
        self.on_iface = np.isin(self.dofs, shared)
        self.iface_pos = np.searchsorted(shared, self.dofs)  # slot in the exchange buffer
        self.niface = shared.size
        self.owned = (first[self.dofs] == rank) & self.free
        self.diag = self._assemble(np.asarray(diag_loc, np.float64), absolute=True)
        self.dinv = np.where(self.free, 1.0 / np.where(self.free, self.diag, 1.0), 0.0)

    # -- communication -------------------------------------------------------
    def _allreduce(self, arr):
        if self.pg is None:
            return arr
        t = self.torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64))
        if self.pg.get_backend() == "nccl":  # NCCL reduces device tensors only
            d = t.to("cuda:%d" % self.torch.cuda.current_device())
            self.pg.all_reduce(d)
            return d.cpu().numpy()
        self.pg.all_reduce(t)
        return t.numpy()

    def _assemble(self, y_loc, absolute=False):
        """Rank-local assemble, then the interface dofs summed over ranks."""
        s = self.sign_r * self.sign_r if absolute else self.sign_r
        out = np.zeros(self.dofs.size)
        np.add.at(out, self.lmap, s * y_loc)
        if self.niface:
            buf = np.zeros(self.niface)
            buf[self.iface_pos[self.on_iface]] = out[self.on_iface]
            buf = self._allreduce(buf)
            out[self.on_iface] = buf[self.iface_pos[self.on_iface]]
        return out

    def _matvec(self, x):
        return self._assemble(self.apply(self.sign_r * x[self.lmap]))

    def _dots(self, *pairs):
        return self._allreduce(np.array([np.sum((a * b)[self.owned]) for a, b in pairs]))

    # -- solve ---------------------------------------------------------------
    def solve(self, b_loc, x0_loc, tol=1e-10, maxit=5000):
        """Rank's local rhs and local Dirichlet values -> rank's local
        solution, iterations. The recurrence and the stopping rule of
        NekLinSysIterCG::DoConjugateGradient (reduced communication)."""
        x0_loc = np.asarray(x0_loc, np.float64)
        r = self._assemble(np.asarray(b_loc, np.float64) - self.apply(x0_loc))
        r[~self.free] = 0.0
        bnorm, eps = self._dots((r, r), (r, r))
        bnorm = bnorm if bnorm > 1e-6 else 1.0
        x = np.zeros(self.dofs.size)
        it = 0
        if eps >= tol * tol * bnorm:
            w = self.dinv * r
            s = self._matvec(w)
            s[~self.free] = 0.0
            rho, mu = self._dots((r, w), (s, w))
            p, q = w.copy(), s.copy()
            alpha, beta, it = rho / mu, 0.0, 1
            while True:
                x += alpha * p
                r -= alpha * q
                w = self.dinv * r
                s = self._matvec(w)
                s[~self.free] = 0.0
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
