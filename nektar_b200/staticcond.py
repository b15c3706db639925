"""Static condensation of the Helmholtz system on the device, the solver of
GlobalLinSysIterativeStaticCond (MultiRegions/GlobalLinSysIterativeStaticCond
.cpp, GlobalLinSysStaticCond.cpp:90-300) with the diagonal preconditioner.

Every element's modes split into boundary modes (vertex, edge and face
modes, which carry the C0 coupling) and interior modes. With the element
matrix K = [[Kbb, Kbi], [Kib, Kii]] the interior unknowns are eliminated
element by element:

    S = Kbb - Kbi Kii^-1 Kib               (Schur complement per element)
    S x_b = b_b - Kbi Kii^-1 b_i           (assembled over the boundary dofs)
    x_i = Kii^-1 (b_i - Kib x_b)           (back substitution per element)

The CG on the condensed system runs on the device exactly as the full one
does (gather fused into the operator, deterministic CSR assemble, Jacobi on
diag(S), graphs), with the Schur blocks as per-element dense operators
(nkb_op_create_dense, an HBM-bound batched GEMV). The element matrices are
taken from the device Helmholtz operators (applied to unit vectors) and the
condensation and the back substitution are done on the host with numpy, as
the reference builds its condensed matrices on the host.
"""
import time

import numpy as np

from .meshgraph import ncoeffs, topology


def boundary_interior(shape, nm):
    """Boundary and interior local mode indices of a shape."""
    verts, edges, faces = topology(shape, nm)
    bnd = set(verts)
    for _, _, lst in edges:
        bnd.update(m for m, _ in lst)
    for _, _, lst in faces:
        bnd.update(m for m, _, _ in lst)
    nc = ncoeffs(shape, nm)
    b = np.array(sorted(bnd), dtype=np.int64)
    i = np.array([m for m in range(nc) if m not in bnd], dtype=np.int64)
    return b, i


def element_matrices(op):
    """K (nelmt, nc, nc) of an Operator: its application to unit vectors."""
    nc, ne = op.in_size // op.nelmt, op.nelmt
    K = np.empty((ne, nc, nc))
    x = np.zeros(ne * nc)
    for j in range(nc):
        x[:] = 0.0
        x[j::nc] = 1.0
        K[:, :, j] = op(x).reshape(ne, nc)
    return K


def condense(K, bm, im):
    """(S, C, Kii_inv, Kib) of element matrices: S = Kbb - C Kib, C = Kbi Kii^-1."""
    Kbb = K[:, bm][:, :, bm]
    Kbi = K[:, bm][:, :, im]
    Kib = K[:, im][:, :, bm]
    Kii_inv = np.linalg.inv(K[:, im][:, :, im])
    C = Kbi @ Kii_inv
    return Kbb - C @ Kib, C, Kii_inv, Kib


class StaticCondSys:
    """Statically condensed Helmholtz system over Helmholtz collection
    operators (Operator) with the C0 map of the full local space."""

    def __init__(self, ops, gmap, nglob, ndir, sign=None, device=0, matrices=None):
        import nektar_b200 as nb
        t0 = time.perf_counter()
        self.ops = list(ops)
        self.parts = []
        gmap = np.asarray(gmap)
        sign = np.ones(gmap.size) if sign is None else np.asarray(sign, dtype=np.float64)
        off = 0
        bglob, bsign = [], []
        for k, op in enumerate(self.ops):
            nc, ne = op.in_size // op.nelmt, op.nelmt
            bm, im = boundary_interior(op.shape, op.nm)
            K = element_matrices(op) if matrices is None else matrices[k]
            S, C, Kii_inv, Kib = condense(K, bm, im)
            gm = gmap[off:off + ne * nc].reshape(ne, nc)
            sg = sign[off:off + ne * nc].reshape(ne, nc)
            bglob.append(gm[:, bm].ravel())
            bsign.append(sg[:, bm].ravel())
            self.parts.append(dict(nc=nc, ne=ne, bm=bm, im=im, S=S, C=C, Kii_inv=Kii_inv,
                                   Kib=Kib, off=off))
            off += ne * nc
        self.nloc = off
        bglob = np.concatenate(bglob)
        # boundary dofs renumbered in their original order (Dirichlet first kept)
        ids = np.unique(bglob)
        if ndir and (ids[:ndir] != np.arange(ndir)).any():
            raise ValueError("Dirichlet dofs must be boundary dofs numbered first")
        renum = np.full(nglob, -1, dtype=np.int64)
        renum[ids] = np.arange(ids.size)
        self.bmap = renum[bglob].astype(np.int32)
        self.bsign = np.concatenate(bsign)
        self.nglob_b, self.ndir = int(ids.size), int(ndir)
        self.nglob = int(nglob)
        self.setup_s = time.perf_counter() - t0
        self.dense = [nb.DenseOperator(p["S"], device=device) for p in self.parts]
        self.sys = nb.GlobalLinSys(self.dense, self.bmap, self.nglob_b, self.ndir,
                                   sign=self.bsign, device=device)

    def condense_rhs(self, b_loc):
        out = []
        for p in self.parts:
            b = np.asarray(b_loc[p["off"]:p["off"] + p["ne"] * p["nc"]]).reshape(p["ne"], p["nc"])
            out.append((b[:, p["bm"]] - np.einsum("ebi,ei->eb", p["C"], b[:, p["im"]])).ravel())
        return np.concatenate(out)

    def solve(self, b_loc, x_loc=None, tol=1e-9, maxit=5000, check_interval=16,
              raise_on_maxit=True):
        """Local rhs and local Dirichlet values -> local solution, report
        (the report's iterations and device time are the condensed CG's)."""
        x_loc = np.zeros(self.nloc) if x_loc is None else np.asarray(x_loc, dtype=np.float64)
        xb0 = np.concatenate([x_loc[p["off"]:p["off"] + p["ne"] * p["nc"]]
                              .reshape(p["ne"], p["nc"])[:, p["bm"]].ravel() for p in self.parts])
        xb, rep = self.sys.solve(self.condense_rhs(b_loc), xb0, tol=tol, maxit=maxit,
                                 check_interval=check_interval, raise_on_maxit=raise_on_maxit)
        x = np.empty(self.nloc)
        ob = 0
        for p in self.parts:
            ne, nc, nbm = p["ne"], p["nc"], p["bm"].size
            b = np.asarray(b_loc[p["off"]:p["off"] + ne * nc]).reshape(ne, nc)
            xbe = xb[ob:ob + ne * nbm].reshape(ne, nbm)
            xie = np.einsum("eij,ej->ei", p["Kii_inv"],
                            b[:, p["im"]] - np.einsum("eib,eb->ei", p["Kib"], xbe))
            xe = x[p["off"]:p["off"] + ne * nc].reshape(ne, nc)
            xe[:, p["bm"]] = xbe
            xe[:, p["im"]] = xie
            ob += ne * nbm
        return x, rep

    def close(self):
        self.sys.close()
        for d in self.dense:
            d.close()
