"""Static condensation on the CPU with the oracle's element matrices: mode
splits, and the condensed system reproduces the full system's solution."""
import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200.staticcond import boundary_interior, condense
from oracle import oracle as O


# interior modes: hex (nm-2)^3; prism (nm-2) * sum_{p=2}^{nm-1} (nm-1-p);
# tet: p >= 2, q >= 1, r >= 1 with p + q + r < nm
@pytest.mark.parametrize("shape,nm,nint", [("hex", 5, 27), ("prism", 6, 24), ("tet", 7, 10)])
def test_boundary_interior_split(shape, nm, nint):
    b, i = boundary_interior(shape, nm)
    from nektar_b200.meshgraph import ncoeffs
    assert i.size == nint and b.size + i.size == ncoeffs(shape, nm)
    assert np.intersect1d(b, i).size == 0


def test_condensed_system_reproduces_full_solution():
    m = nb.BoxMesh("hex", 3, 5, 6, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    T = dict(m.T)
    T["w"] = m.T["ws"]
    nc, ne = m.nc, m.nelmt
    K = np.zeros((ne, nc, nc))
    for j in range(nc):
        x = np.zeros(ne * nc)
        x[j::nc] = 1.0
        K[:, :, j] = O.helmholtz("hex", 5, m.nq, ne, T, m.jac, m.df, x, 1.3, True).reshape(ne, nc)
    gm = gmap.reshape(ne, nc)
    G = np.zeros((nglob, nglob))
    for e in range(ne):
        np.add.at(G, (gm[e][:, None], gm[e][None, :]), K[e])
    rng = np.random.default_rng(2)
    b_loc = rng.uniform(-1, 1, ne * nc)
    b = np.zeros(nglob)
    np.add.at(b, gmap, b_loc)
    x_full = np.linalg.solve(G[ndir:, ndir:], b[ndir:])
    bm, im = boundary_interior("hex", 5)
    S, C, Kii_inv, Kib = condense(K, bm, im)
    bl = b_loc.reshape(ne, nc)
    bc = bl[:, bm] - np.einsum("ebi,ei->eb", C, bl[:, im])
    gb = gm[:, bm]
    ids = np.unique(gb)
    renum = np.full(nglob, -1)
    renum[ids] = np.arange(ids.size)
    gbr = renum[gb]
    Gs = np.zeros((ids.size, ids.size))
    for e in range(ne):
        np.add.at(Gs, (gbr[e][:, None], gbr[e][None, :]), S[e])
    rb = np.zeros(ids.size)
    np.add.at(rb, gbr.ravel(), bc.ravel())
    xb = np.concatenate([np.zeros(ndir), np.linalg.solve(Gs[ndir:, ndir:], rb[ndir:])])
    xbl = xb[gbr]
    xil = np.einsum("eij,ej->ei", Kii_inv, bl[:, im] - np.einsum("eib,eb->ei", Kib, xbl))
    xg = np.concatenate([np.zeros(ndir), x_full])
    scale = np.abs(xg).max()  # two dense solves agree to rounding times the conditioning
    assert np.abs(xg[gm[:, bm]] - xbl).max() < 1e-10 * scale
    assert np.abs(xg[gm[:, im]] - xil).max() < 1e-10 * scale
