"""Mixed-element meshes: a box grid of n^3 cells in which a seeded permutation
keeps some cells as hexes and splits others into 2 prisms or 6 tets, with a
polynomial order drawn per cell, all curved by the box map. Elements are
grouped into one collection per (shape, P) -- the reference's grouping by
basis key (MultiRegions/ExpList.cpp:5930) -- and a `Batch` applies every
collection's operator in one call.

The prisms and tets of one split cell share the cell's order (a conforming
choice; orders are drawn per cell, not per element).
"""
import numpy as np

SHAPE_ORDER = ("hex", "prism", "tet")


class MixedMesh:
    def __init__(self, n=40, ncells=(20000, 15000, 10000), pmin=2, pmax=10, amp=0.05, seed=0):
        """ncells: cells kept as hexes, split into prisms, split into tets."""
        if sum(ncells) > n ** 3:
            raise ValueError("more cells requested than the %d^3 grid has" % n)
        rng = np.random.default_rng(seed)
        perm = rng.permutation(n ** 3)
        bounds = np.cumsum((0,) + tuple(ncells))
        self.n, self.amp, self.seed = n, amp, seed
        self.cell_p = {}
        self.groups = []  # (shape, P, sorted cell ids)
        for s, shape in enumerate(SHAPE_ORDER):
            cells = perm[bounds[s]:bounds[s + 1]]
            P = rng.integers(pmin, pmax + 1, len(cells))
            for p in range(pmin, pmax + 1):
                sel = np.sort(cells[P == p]).astype(np.int32)
                if len(sel):
                    self.groups.append((shape, int(p), sel))

    def meshes(self):
        """One nektar_b200.BoxMesh per collection, in group order."""
        import nektar_b200 as nb
        for shape, p, cells in self.groups:
            yield nb.BoxMesh(shape, self.n, p + 1, p + 2, amp=self.amp, cells=cells)

    def collections(self, optype="helmholtz", lam=1.0, device=0, keep_geometry=False):
        """(mesh, operator) per collection; the host geometry is dropped once
        the operator holds its device copy unless keep_geometry."""
        import nektar_b200 as nb
        out = []
        for m in self.meshes():
            op = nb.Operator(optype, m, device=device)
            if optype == "helmholtz":
                op.set_factors(lam)
            if not keep_geometry:
                m.jac = m.df = None
            out.append((m, op))
        return out
