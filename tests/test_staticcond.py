"""Static condensation on the CPU with the oracle's element matrices: mode
splits, and the condensed system reproduces the full system's solution."""
import os

import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200.staticcond import boundary_interior, condense
from oracle import oracle as O
from tests.helpers import ref_path


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


def test_reference_helmholtz_energy():
    """The low-energy reference element is the unit cube: the constant
    function has energy lambda, the function x has 1 + lambda / 3."""
    from nektar_b200.meshgraph import topology
    from nektar_b200.staticcond import reference_helmholtz
    lam, nm = 2.5, 6
    K = reference_helmholtz("hex", nm, lam)
    assert np.abs(K - K.T).max() < 1e-13
    verts = topology("hex", nm)[0]
    one = np.zeros(nm ** 3)
    one[verts] = 1.0
    x = np.zeros(nm ** 3)
    x[[verts[i] for i in (1, 2, 5, 6)]] = 1.0  # the vertices at x = 1
    assert abs(one @ K @ one - lam) < 1e-12
    assert abs(x @ K @ x - (1.0 + lam / 3.0)) < 1e-12


def test_lowenergy_transform_decouples_reference_element():
    """R S of the reference element has no coupling of a vertex to the
    interior modes of its edges and faces, nor of an edge to its faces."""
    from nektar_b200.staticcond import (_entities, lowenergy_transform, reference_helmholtz)
    nm = 6
    bm, im = boundary_interior("hex", nm)
    S = condense(reference_helmholtz("hex", nm, 1.0)[None], bm, im)[0][0]
    R = lowenergy_transform("hex", nm, S)
    V, E, F, ev, fv = _entities("hex", nm, bm)
    RS = R @ S
    assert np.allclose(np.diag(R), 1.0)
    for v, pv in enumerate(V):
        cols = np.concatenate([E[e] for e, (a, b) in enumerate(ev) if v in (a, b)] +
                              [F[f] for f in range(6) if v in fv[f]])
        assert np.abs(RS[pv, cols]).max() < 1e-12 * np.abs(S).max()
    for e, (a, b) in enumerate(ev):
        cols = np.concatenate([F[f] for f in range(6) if a in fv[f] and b in fv[f]])
        assert np.abs(RS[np.ix_(E[e], cols)]).max() < 1e-12 * np.abs(S).max()


def _oracle_matrices(shape, nm, nq, ne, T, jac, df, lam):
    from nektar_b200.meshgraph import ncoeffs
    To = dict(T)
    To["w"] = T["ws"]
    nc = ncoeffs(shape, nm)
    K = np.zeros((ne, nc, nc))
    for j in range(nc):
        x = np.zeros(ne * nc)
        x[j::nc] = 1.0
        K[:, :, j] = O.helmholtz(shape, nm, nq, ne, To, jac, df, x, lam, True).reshape(ne, nc)
    return K


def _oracle_reference_R(shape, nm, lam):
    """The low-energy transform with the oracle's reference element matrix."""
    from nektar_b200.staticcond import lowenergy_transform, reference_geometry
    T, nq, jac, df = reference_geometry(shape, nm)
    Kr = _oracle_matrices(shape, nm, nq, 1, T, jac, df, lam)
    bm, im = boundary_interior(shape, nm)
    return lowenergy_transform(shape, nm, condense(Kr, bm, im)[0][0])


def _rotated_hex_condensed(nm=5, n=3, lam=1.3, shape="hex"):
    """Condensed matrices of a session with rotated element frames (so the
    map carries signs), from the oracle's element matrices."""
    from nektar_b200.meshgraph import SessionMesh, ncoeffs
    from nektar_b200.session import read_session, write_box_session, write_hex_box_session
    if shape == "hex":
        s = read_session(write_hex_box_session(n, nm, lam, "x", "0", "x", shuffle_seed=4))
    else:
        s = read_session(write_box_session(shape, n, nm, lam, "x", "0", "x", shuffle_seed=4))
    mesh = SessionMesh(s)
    c = mesh.collections[0]
    ne, nc = c.nelmt, ncoeffs(shape, nm)
    K = _oracle_matrices(shape, nm, c.nq, ne, c.T, c.jac, c.df, lam)
    bm, im = boundary_interior(shape, nm)
    S, C, Kii_inv, Kib = condense(K, bm, im)
    gm = np.asarray(mesh.gmap).reshape(ne, nc)
    sg = np.asarray(mesh.sign, dtype=np.float64).reshape(ne, nc)
    ids = np.unique(gm[:, bm])
    renum = np.full(mesh.nglob, -1)
    renum[ids] = np.arange(ids.size)
    return dict(S=S, bm=bm, im=im, ne=ne, nm=nm, lam=lam, shape=shape,
                bmap=renum[gm[:, bm]].ravel(), bsign=sg[:, bm].ravel(), nb=ids.size,
                ndir=mesh.ndir, K=K, C=C, Kii_inv=Kii_inv, Kib=Kib, gm=gm, sg=sg,
                nglob=mesh.nglob)


def _assemble(mats, bmap, bsign, nb):
    ne, n, _ = mats.shape
    G = np.zeros((nb, nb))
    gm, sg = bmap.reshape(ne, n), bsign.reshape(ne, n)
    for e in range(ne):
        np.add.at(G, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * sg[e][None, :] * mats[e])
    return G


def test_lowenergy_basis_is_conforming():
    """The condensed system solved in the low-energy basis (S~ = R S R^T per
    element, right-hand side R b, solution R^T x~) gives the solution of the
    original condensed system: the reference-element transform is the same
    function space on a mesh whose elements meet in rotated frames."""
    from nektar_b200.staticcond import lowenergy_transform, reference_helmholtz
    d = _rotated_hex_condensed()
    S, ne, nd = d["S"], d["ne"], d["ndir"]
    nbm = d["bm"].size
    Sr = condense(reference_helmholtz("hex", d["nm"], d["lam"])[None], d["bm"], d["im"])[0][0]
    R = lowenergy_transform("hex", d["nm"], Sr)
    rng = np.random.default_rng(7)
    gm, sg = d["bmap"].reshape(ne, nbm), d["bsign"].reshape(ne, nbm)
    xg = np.zeros(d["nb"])
    xg[:nd] = rng.uniform(-1, 1, nd)           # Dirichlet values
    b_loc = rng.uniform(-1, 1, (ne, nbm))
    x0 = np.where(gm < nd, sg * xg[gm], 0.0)   # local Dirichlet values

    def solve(mats, b, x0l):
        G = _assemble(mats, d["bmap"], d["bsign"], d["nb"])
        r = np.zeros(d["nb"])
        np.add.at(r, gm.ravel(), (sg * (b - np.einsum("eij,ej->ei", mats, x0l))).ravel())
        x = np.zeros(d["nb"])
        x[nd:] = np.linalg.solve(G[nd:, nd:], r[nd:])
        return x0l + sg * x[gm]

    x_ref = solve(S, b_loc, x0)
    x_le = solve(R @ S @ R.T, b_loc @ R.T, x0 @ np.linalg.inv(R)) @ R
    assert np.abs(x_le - x_ref).max() < 1e-10 * np.abs(x_ref).max()
    # local Dirichlet values that differ between the elements sharing a dof
    # (as a per-face boundary projection can leave them) stay on the
    # Dirichlet modes: the free modes match the original basis's solve
    x0b = x0 + np.where(gm < nd, rng.uniform(-1e-3, 1e-3, x0.shape), 0.0)
    x_ref = solve(S, b_loc, x0b)
    x_le = solve(R @ S @ R.T, b_loc @ R.T, x0b @ np.linalg.inv(R)) @ R
    assert np.abs(x_le - x_ref).max() < 1e-10 * np.abs(x_ref).max()


def _precon_matrix(blocks, diag, nd):
    """Dense preconditioner: inverse blocks, Jacobi elsewhere (free dofs)."""
    M = np.diag(1.0 / diag)
    for dofs, inv in blocks:
        f = np.asarray(dofs) - nd
        M[np.ix_(f, f)] = inv
    return M


def test_block_and_lowenergy_preconditioners_condition_number():
    """Condition numbers of the preconditioned condensed systems: Block
    below Jacobi, LowEnergy well below both (the order of the reference's
    Diagonal / Block / LowEnergy preconditioners)."""
    from nektar_b200.staticcond import (entity_blocks, lowenergy_transform, reference_helmholtz)
    d = _rotated_hex_condensed(nm=6, n=3)
    nd = d["ndir"]
    Sr = condense(reference_helmholtz("hex", d["nm"], d["lam"])[None], d["bm"], d["im"])[0][0]
    R = lowenergy_transform("hex", d["nm"], Sr)
    kappa = {}
    for name, S in (("jacobi", d["S"]), ("block", d["S"]), ("lowenergy", R @ d["S"] @ R.T)):
        A = _assemble(S, d["bmap"], d["bsign"], d["nb"])[nd:, nd:]
        if name == "jacobi":
            M = np.diag(1.0 / np.diag(A))
        else:
            part = dict(S=S, ne=d["ne"], bm=d["bm"], shape="hex", nm=d["nm"])
            blocks = entity_blocks([part], d["bmap"], d["bsign"], nd)
            M = _precon_matrix(blocks, np.diag(A), nd)
            for dofs, inv in blocks:  # each block is the assembled matrix's own block
                f = np.asarray(dofs) - nd
                assert np.allclose(np.linalg.inv(inv), A[np.ix_(f, f)], rtol=1e-10, atol=1e-12)
        L = np.linalg.cholesky(M)
        ev = np.linalg.eigvalsh(L.T @ A @ L)
        kappa[name] = ev[-1] / ev[0]
    assert kappa["block"] < kappa["jacobi"]
    assert kappa["lowenergy"] < 0.25 * kappa["block"]


def test_solve_maps_reproduce_full_solution():
    """The per-element maps around the condensed CG (W: condensed and
    low-energy transformed right-hand side; V: back to the local modes with
    the interior back substitution) give the full system's solution."""
    from nektar_b200.staticcond import lowenergy_transform, reference_helmholtz, solve_maps
    d = _rotated_hex_condensed(nm=5, n=2)
    ne, nd, nc = d["ne"], d["ndir"], d["nm"] ** 3
    nbm = d["bm"].size
    gm, sg = d["gm"], d["sg"]
    rng = np.random.default_rng(5)
    b_loc = rng.uniform(-1, 1, (ne, nc))
    G = np.zeros((d["nglob"], d["nglob"]))
    for e in range(ne):
        np.add.at(G, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * sg[e][None, :] * d["K"][e])
    bg = np.zeros(d["nglob"])
    np.add.at(bg, gm.ravel(), (sg * b_loc).ravel())
    xg = np.zeros(d["nglob"])
    xg[nd:] = np.linalg.solve(G[nd:, nd:], bg[nd:])
    x_full = sg * xg[gm]
    Sr = condense(reference_helmholtz("hex", d["nm"], d["lam"])[None], d["bm"], d["im"])[0][0]
    for R in (None, lowenergy_transform("hex", d["nm"], Sr)):
        W, V = solve_maps(d["C"], d["Kii_inv"], d["Kib"], d["bm"], d["im"], R)
        St = d["S"] if R is None else R @ d["S"] @ R.T
        bt = np.einsum("ebc,ec->eb", W, b_loc)
        A = _assemble(St, d["bmap"], d["bsign"], d["nb"])
        gb, sb = d["bmap"].reshape(ne, nbm), d["bsign"].reshape(ne, nbm)
        r = np.zeros(d["nb"])
        np.add.at(r, gb.ravel(), (sb * bt).ravel())
        xt = np.zeros(d["nb"])
        xt[nd:] = np.linalg.solve(A[nd:, nd:], r[nd:])
        z = np.concatenate([sb * xt[gb], b_loc[:, d["im"]]], axis=1)
        x = np.einsum("ecz,ez->ec", V, z)
        assert np.abs(x - x_full).max() < 1e-10 * np.abs(x_full).max()


def test_reference_cube_matches_oracle():
    """The host-built reference cube matrix equals the oracle's Helmholtz
    matrix of the same element (affine unit cube, nm+1 GLL points)."""
    from nektar_b200.staticcond import reference_geometry, reference_helmholtz
    nm, lam = 6, 0.7
    T, nq, jac, df = reference_geometry("hex", nm)
    Ko = _oracle_matrices("hex", nm, nq, 1, T, jac, df, lam)[0]
    Kr = reference_helmholtz("hex", nm, lam)
    assert np.abs(Kr - Ko).max() < 1e-13 * np.abs(Ko).max()


@pytest.mark.parametrize("nm", [5, 7])
def test_tet_lowenergy_is_conforming_and_preconditions(nm):
    """Tetrahedral meshes: the regular-tetrahedron transform gives a
    conforming basis on a tet session (faces shared in different local
    frames) and cuts the condition number of the block-preconditioned
    condensed system well below Jacobi's."""
    from nektar_b200.staticcond import entity_blocks
    d = _rotated_hex_condensed(nm=nm, n=2, shape="tet")
    S, ne, nd = d["S"], d["ne"], d["ndir"]
    nbm = d["bm"].size
    R = _oracle_reference_R("tet", nm, d["lam"])
    gm, sg = d["bmap"].reshape(ne, nbm), d["bsign"].reshape(ne, nbm)
    rng = np.random.default_rng(8)
    b = rng.uniform(-1, 1, (ne, nbm))

    def solve(mats, bb):
        G = _assemble(mats, d["bmap"], d["bsign"], d["nb"])
        r = np.zeros(d["nb"])
        np.add.at(r, gm.ravel(), (sg * bb).ravel())
        x = np.zeros(d["nb"])
        x[nd:] = np.linalg.solve(G[nd:, nd:], r[nd:])
        return sg * x[gm]

    x_ref = solve(S, b)
    x_le = solve(R @ S @ R.T, b @ R.T) @ R
    assert np.abs(x_le - x_ref).max() < 1e-10 * np.abs(x_ref).max()
    kappa = {}
    for name, mats in (("jacobi", S), ("lowenergy", R @ S @ R.T)):
        A = _assemble(mats, d["bmap"], d["bsign"], d["nb"])[nd:, nd:]
        if name == "jacobi":
            M = np.diag(1.0 / np.diag(A))
        else:
            part = dict(S=mats, ne=ne, bm=d["bm"], shape="tet", nm=nm)
            M = _precon_matrix(entity_blocks([part], d["bmap"], d["bsign"], nd), np.diag(A), nd)
        L = np.linalg.cholesky(M)
        ev = np.linalg.eigvalsh(L.T @ A @ L)
        kappa[name] = ev[-1] / ev[0]
    assert kappa["lowenergy"] < 0.5 * kappa["jacobi"]


def _oracle_reference(shape, nm, lam):
    from nektar_b200.staticcond import reference_geometry
    T, nq, jac, df = reference_geometry(shape, nm)
    return _oracle_matrices(shape, nm, nq, 1, T, jac, df, lam)[0]


def _session_parts(shape, nm, n, lam, seed):
    """Per-collection condensed matrices of a box session (oracle element
    matrices) with the boundary map over all collections."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session, write_box_session
    s = read_session(write_box_session(shape, n, nm, lam, "x", "0", "x", shuffle_seed=seed))
    mesh = SessionMesh(s)
    parts, bg, bs = [], [], []
    for c, off in zip(mesh.collections, mesh.offsets):
        K = _oracle_matrices(c.shape, nm, c.nq, c.nelmt, c.T, c.jac, c.df, lam)
        bm, im = boundary_interior(c.shape, nm)
        S = condense(K, bm, im)[0]
        gm = np.asarray(mesh.gmap[off:off + c.nelmt * c.nc]).reshape(c.nelmt, c.nc)
        sg = np.asarray(mesh.sign[off:off + c.nelmt * c.nc], dtype=np.float64).reshape(
            c.nelmt, c.nc)
        parts.append(dict(S=S, ne=c.nelmt, bm=bm, shape=c.shape, nm=nm))
        bg.append(gm[:, bm].ravel())
        bs.append(sg[:, bm].ravel())
    bg = np.concatenate(bg)
    ids = np.unique(bg)
    renum = np.full(mesh.nglob, -1)
    renum[ids] = np.arange(ids.size)
    return parts, renum[bg], np.concatenate(bs), ids.size, mesh.ndir


@pytest.mark.parametrize("shape", ["prism", "hexprism"])
def test_prism_lowenergy_is_conforming_and_preconditions(shape):
    """Prisms (alone and meeting hexahedra): the prism transform assembled
    from the hexahedron's and the tetrahedron's entries still describes a
    conforming basis, and the block-preconditioned system is far better
    conditioned than with Jacobi."""
    from nektar_b200.staticcond import entity_blocks, lowenergy_transforms
    nm, lam = 6, 1.3
    parts, bmap, bsign, nb, nd = _session_parts(shape, nm, 2, lam, 6)
    Rs = lowenergy_transforms({p["shape"] for p in parts}, nm, lam, reference=_oracle_reference)
    rng = np.random.default_rng(9)

    def assemble(mats_list):
        G = np.zeros((nb, nb))
        ob = 0
        for p, mats in zip(parts, mats_list):
            k = p["ne"] * p["bm"].size
            G += _assemble(mats, bmap[ob:ob + k], bsign[ob:ob + k], nb)
            ob += k
        return G

    bl = [rng.uniform(-1, 1, (p["ne"], p["bm"].size)) for p in parts]

    def solve(mats_list, b_list):
        G = assemble(mats_list)
        r = np.zeros(nb)
        ob, out = 0, []
        for p, bb in zip(parts, b_list):
            k = p["ne"] * p["bm"].size
            np.add.at(r, bmap[ob:ob + k], bsign[ob:ob + k] * bb.ravel())
            ob += k
        x = np.zeros(nb)
        x[nd:] = np.linalg.solve(G[nd:, nd:], r[nd:])
        ob = 0
        for p in parts:
            k = p["ne"] * p["bm"].size
            out.append((bsign[ob:ob + k] * x[bmap[ob:ob + k]]).reshape(p["ne"], -1))
            ob += k
        return out

    x_ref = solve([p["S"] for p in parts], bl)
    St = [Rs[p["shape"]] @ p["S"] @ Rs[p["shape"]].T for p in parts]
    x_le = solve(St, [bb @ Rs[p["shape"]].T for p, bb in zip(parts, bl)])
    scale = max(np.abs(x).max() for x in x_ref)
    for p, xr, xl in zip(parts, x_ref, x_le):
        assert np.abs(xl @ Rs[p["shape"]] - xr).max() < 1e-10 * scale
    kappa = {}
    for name, mats in (("jacobi", [p["S"] for p in parts]), ("lowenergy", St)):
        A = assemble(mats)[nd:, nd:]
        if name == "jacobi":
            M = np.diag(1.0 / np.diag(A))
        else:
            tp = [dict(p, S=m) for p, m in zip(parts, mats)]
            M = _precon_matrix(entity_blocks(tp, bmap, bsign, nd), np.diag(A), nd)
        L = np.linalg.cholesky(M)
        ev = np.linalg.eigvalsh(L.T @ A @ L)
        kappa[name] = ev[-1] / ev[0]
    assert kappa["lowenergy"] < 0.5 * kappa["jacobi"]


def _gauss_jordan_colmajor(M):
    """The in-place Gauss-Jordan inversion of nkb_blocks_invert (no pivoting,
    normalised pivot row, column k stashed before the update), then the
    transpose it ends with."""
    M = M.copy()
    n = M.shape[0]
    for k in range(n):
        pinv = 1.0 / M[k, k]
        col = M[:, k].copy()
        row = M[k, :] * pinv
        row[k] = pinv
        upd = M.copy()
        upd[:, k] = 0.0
        M = upd - np.outer(col, row)
        M[k, :] = row
    return M.T


@pytest.mark.parametrize("case", ["hex", "prism", "hexprism"])
def test_device_block_inputs_reproduce_entity_blocks(case):
    """What the device builds the Block / LowEnergy blocks from: the
    contribution arrays (blocks, elements, rows in block order, signs),
    summed in their order as nkb_blocks_accumulate does, and inverted as
    nkb_blocks_invert does, give entity_blocks' inverses, in the column-major
    layout that nkb_sys_set_blocks takes."""
    from nektar_b200.staticcond import contribution_arrays, entity_blocks, entity_index
    if case == "hex":
        d = _rotated_hex_condensed(nm=6, n=3)
        parts = [dict(S=d["S"], ne=d["ne"], bm=d["bm"], shape="hex", nm=d["nm"])]
        bmap, bsign, nd = d["bmap"], d["bsign"], d["ndir"]
    else:
        parts, bmap, bsign, _, nd = _session_parts(case, 5, 2, 1.3, 6)
    dofs, contrib = entity_index(parts, bmap, bsign, nd)
    ref = entity_blocks(parts, bmap, bsign, nd)
    assert len(ref) == len(dofs) > 0
    sizes = np.array([x.size for x in dofs])
    A = [np.zeros((n, n)) for n in sizes]
    for p, entries in zip(parts, contrib):
        if not entries:
            continue
        cptr, celm, cloc, csgn = contribution_arrays(entries, len(dofs))
        assert cptr[0] == 0 and cptr[-1] == celm.size and (np.diff(cptr) >= 0).all()
        off = 0
        for b in range(len(dofs)):
            n = sizes[b]
            for c in range(cptr[b], cptr[b + 1]):
                l, sg = cloc[off:off + n], csgn[off:off + n].astype(np.float64)
                A[b] += np.outer(sg, sg) * p["S"][celm[c]][np.ix_(l, l)]
                off += n
        assert off == cloc.size
    for (rd, rinv), dd, a in zip(ref, dofs, A):
        assert np.array_equal(rd, dd)
        inv_cm = _gauss_jordan_colmajor(a)
        assert np.allclose(inv_cm.T, rinv, rtol=1e-10, atol=1e-13 * np.abs(rinv).max())


@pytest.mark.parametrize("shape,nmax,nm", [("hex", 6, 4), ("tet", 7, 5), ("prism", 6, 3)])
def test_transform_of_order_is_the_highest_order_transform_cut_down(shape, nmax, nm):
    """ExtractLocMat: the transform of an element of lower order holds the
    highest order's entries between the modes with the same vertex, edge or
    face and polynomial indices, a unit diagonal and nothing else."""
    from nektar_b200.staticcond import boundary_keys, transform_of_order
    R = _oracle_reference_R("tet" if shape == "tet" else "hex", nmax, 1.1)
    if shape == "prism":  # any matrix of the prism's size exercises the cut
        nbp = boundary_interior("prism", nmax)[0].size
        R = np.eye(nbp) + np.triu(np.random.default_rng(2).uniform(-1, 1, (nbp, nbp)), 1)
    kmax, klo = boundary_keys(shape, nmax), boundary_keys(shape, nm)
    assert len(klo) == boundary_interior(shape, nm)[0].size and set(klo) <= set(kmax)
    Rl = transform_of_order(shape, nm, nmax, R)
    pos = {k: i for i, k in enumerate(kmax)}
    for i, ki in enumerate(klo):
        for j, kj in enumerate(klo):
            assert Rl[i, j] == R[pos[ki], pos[kj]]
    assert transform_of_order(shape, nmax, nmax, R) is R


def _lowenergy_condensed(s, lam, Ks=None):
    """A session's mesh condensed on the host with the oracle's element
    matrices (or Ks) through the library's own LowEnergy set-up functions
    (condensed_parts, boundary_map, lowenergy_part_transforms,
    element_transforms, solve_maps)."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.staticcond import (boundary_map, condensed_parts, element_transforms,
                                        lowenergy_part_transforms, solve_maps)
    m = SessionMesh(s)
    cols = m.collections
    parts = condensed_parts([(c.shape, c.nm, c.nelmt) for c in cols])
    bmap, bsign, nb_ = boundary_map(parts, m.gmap, m.sign, m.nglob, m.ndir)
    lowenergy_part_transforms(parts, bsign, lam,
                              reference=lambda sh, n, lm: _oracle_reference(sh, n, lm))
    if Ks is None:
        Ks = [_oracle_matrices(c.shape, c.nm, c.nq, c.nelmt, c.T, c.jac, c.df, lam) for c in cols]
    for K, p in zip(Ks, parts):
        S, C, Kii_inv, Kib = condense(K, p["bm"], p["im"])
        Re = element_transforms(p)
        p["S0"], p["S"] = S, Re @ S @ np.swapaxes(Re, -1, -2)
        p["W"], p["V"] = solve_maps(C, Kii_inv, Kib, p["bm"], p["im"], Re)
    return dict(m=m, parts=parts, Ks=Ks, bmap=bmap, bsign=bsign, nb=nb_)


def _lowenergy_solve(d, b, x0):
    """(local solution, assembled S~, assembled S) of the condensed
    low-energy system with a dense solve in place of the CG, step by step
    as StaticCondSys.solve runs it: b~ = W b, the local Dirichlet values
    lifted with R^-T, the boundary solve, and V back to the local modes."""
    m, parts, bmap, bsign, nb_ = d["m"], d["parts"], d["bmap"], d["bsign"], d["nb"]
    nd = m.ndir
    A = np.zeros((nb_, nb_))
    A0 = np.zeros((nb_, nb_))  # the condensed system in the original basis
    rb = np.zeros(nb_)
    ob, xb0s = 0, []
    for p in parts:
        ne, nbm = p["ne"], p["bm"].size
        sl = slice(p["off"], p["off"] + ne * p["nc"])
        be = b[sl].reshape(ne, -1)
        xb0 = x0[sl].reshape(ne, -1)[:, p["bm"]] @ p["Rinv"]
        gm, sg = bmap[ob:ob + ne * nbm].reshape(ne, nbm), bsign[ob:ob + ne * nbm].reshape(ne, nbm)
        for e in range(ne):
            for M, Se in ((A, p["S"][e]), (A0, p["S0"][e])):
                np.add.at(M, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * Se * sg[e][None, :])
        rl = np.einsum("eij,ej->ei", p["W"], be) - np.einsum("eij,ej->ei", p["S"], xb0)
        np.add.at(rb, gm.ravel(), (sg * rl).ravel())
        xb0s.append(xb0)
        ob += ne * nbm
    xt = np.zeros(nb_)
    xt[nd:] = np.linalg.solve(A[nd:, nd:], rb[nd:])
    x = np.empty(m.nloc)
    ob = 0
    for p, xb0 in zip(parts, xb0s):
        ne, nbm = p["ne"], p["bm"].size
        sl = slice(p["off"], p["off"] + ne * p["nc"])
        xe = xb0 + bsign[ob:ob + ne * nbm].reshape(ne, nbm) * xt[bmap[ob:ob + ne * nbm]].reshape(
            ne, nbm)
        z = np.concatenate([xe, b[sl].reshape(ne, -1)[:, p["im"]]], axis=1)
        x[sl] = np.einsum("eij,ej->ei", p["V"], z).ravel()
        ob += ne * nbm
    return x, A, A0


@pytest.mark.parametrize("shape,orders", [("tet", [3, 4, 5, 6]), ("hex", [4, 6, 5]),
                                          ("prism", [4, 6, 5]), ("hexprism", [5, 3, 4])])
def test_variable_order_lowenergy_solve_matches_full_solve(shape, orders):
    """Meshes of variable order (the reference's *_VarP_iterLE sessions):
    the transforms cut from the highest order, with the modes a lower-order
    neighbour lacks masked (S~ = R M S M R^T, b~ = R M b, x = M R^T x~; the
    Dirichlet values lifted with the unmasked R^-T), give the full system's
    solution; the entity blocks are the assembled S~'s own blocks over the
    modes of nonzero sign, and they precondition it better than Jacobi."""
    from nektar_b200.session import read_session, with_orders, write_box_session
    from nektar_b200.staticcond import entity_blocks
    lam = 1.3
    s = read_session(with_orders(write_box_session(shape, 2, max(orders), lam, "x", "0", "x",
                                                   shuffle_seed=3), orders, seed=1))
    d = _lowenergy_condensed(s, lam)
    m, parts = d["m"], d["parts"]
    assert any(p["mask"] is not None for p in parts)
    nd = m.ndir
    rng = np.random.default_rng(5)
    b = rng.uniform(-1, 1, m.nloc)
    x0 = m.dirichlet_local()
    # the full system (dense, with the local lifting of the device CG)
    G = np.zeros((m.nglob, m.nglob))
    r = np.zeros(m.nglob)
    for p, K in zip(parts, d["Ks"]):
        sl = slice(p["off"], p["off"] + p["ne"] * p["nc"])
        gm, sg = m.gmap[sl].reshape(p["ne"], p["nc"]), m.sign[sl].reshape(p["ne"], p["nc"])
        for e in range(p["ne"]):
            np.add.at(G, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * K[e] * sg[e][None, :])
        np.add.at(r, gm.ravel(), (sg * (b[sl].reshape(p["ne"], -1) -
                                        np.einsum("eij,ej->ei", K, x0[sl].reshape(p["ne"], -1))))
                  .ravel())
    xg = np.zeros(m.nglob)
    xg[nd:] = np.linalg.solve(G[nd:, nd:], r[nd:])
    x_full = x0 + m.sign * xg[m.gmap]
    x_le, A, A0 = _lowenergy_solve(d, b, x0)
    assert np.abs(x_le - x_full).max() < 1e-10 * np.abs(x_full).max()
    # entity blocks over the active modes: the assembled matrix's own blocks
    blocks = entity_blocks(parts, d["bmap"], d["bsign"], nd)
    assert blocks
    Af = A[nd:, nd:]
    for dofs, inv in blocks:
        f = np.asarray(dofs) - nd
        assert np.allclose(np.linalg.inv(inv), Af[np.ix_(f, f)], rtol=1e-10, atol=1e-12)
    kappa = {}
    A0f = A0[nd:, nd:]
    for name, M, Am in (("jacobi", np.diag(1.0 / np.diag(A0f)), A0f),
                        ("lowenergy", _precon_matrix(blocks, np.diag(Af), nd), Af)):
        L = np.linalg.cholesky(M)
        ev = np.linalg.eigvalsh(L.T @ Am @ L)
        kappa[name] = ev[-1] / ev[0]
    # measured: hex 104 -> 9.6, prism 134 -> 15.9, hexprism 39 -> 11.7, and on
    # the 48 tetrahedra (186 free dofs) 28.7 -> 17.2
    assert kappa["lowenergy"] < 0.65 * kappa["jacobi"], kappa


_REF_TET_VARP = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Tet_VarP.xml")


@pytest.mark.skipif(not os.path.exists(_REF_TET_VARP), reason="reference tree not mounted")
def test_reference_tet_varp_lowenergy_session_reproduces_its_record():
    """Helmholtz3D_CG_Tet_VarP_iterLE.tst (-I GlobalSysSoln=IterativeStaticCond
    -I Preconditioner=LowEnergyBlock on the orders 3-6 tetrahedral session):
    the condensed low-energy system of the library's set-up, solved densely,
    gives the recorded L2 0.00416454 (tolerance 1e-7) and Linf 0.0313733
    (tolerance 1e-6)."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session
    from tests.session_oracle import oracle_errors, oracle_system
    s = read_session(_REF_TET_VARP)
    lam = float(s.parameters["Lambda"])
    Ks, b_loc, robin = oracle_system(s, SessionMesh(s))
    assert not robin
    d = _lowenergy_condensed(s, lam, Ks)
    assert len({p["nm"] for p in d["parts"]}) == 4 and any(p["mask"] is not None
                                                          for p in d["parts"])
    x, _, _ = _lowenergy_solve(d, b_loc, d["m"].dirichlet_local())
    linf, l2 = oracle_errors(s, d["m"], x)
    printed = lambda v: float("%g" % v)  # noqa: E731  (the demo prints six digits)
    assert abs(printed(l2) - 0.00416454) < 1e-7 and abs(printed(linf) - 0.0313733) < 1e-6


def test_mask_groups_cover_every_element_once_with_its_own_transform():
    """The device set-up condenses each group of elements that share a
    variable-order mask with one transform: the groups partition the
    elements, and each group's transform is every member's R M_e."""
    from nektar_b200.session import read_session, with_orders, write_box_session
    from nektar_b200.staticcond import _mask_groups, element_transforms
    s = read_session(with_orders(write_box_session("tet", 2, 5, 1.0, "x", "0", "x",
                                                   shuffle_seed=3), [3, 5, 4], seed=1))
    d = _lowenergy_condensed(s, 1.0)
    masked = [p for p in d["parts"] if p["mask"] is not None]
    assert masked
    for p in d["parts"]:
        groups = _mask_groups(p)
        if p["mask"] is None:
            assert len(groups) == 1 and groups[0][0] is None and groups[0][1] is p["R"]
            continue
        rows = np.concatenate([r for r, _ in groups])
        assert np.array_equal(np.sort(rows), np.arange(p["ne"]))
        Re = element_transforms(p)
        for r, R in groups:
            assert np.array_equal(Re[r], np.broadcast_to(R, (r.size,) + R.shape))


_REF_PRISM = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Prism.xml")


@pytest.mark.skipif(not os.path.exists(_REF_PRISM), reason="reference tree not mounted")
def test_reference_prism_lowenergy_session_reproduces_its_record():
    """Helmholtz3D_CG_Prism_VarP_iterLE.tst (-I GlobalSysSoln=IterativeStaticCond
    -I Preconditioner=LowEnergyBlock on the Prism session): the prism
    transform assembled from the cube's and the tetrahedron's entries
    (ReSetPrismMaxRMat) keeps the basis conforming on the reference's own
    mesh, so the condensed low-energy solve gives the recorded L2 0.000385246
    and Linf 0.00539787 (tolerance 1e-9)."""
    from nektar_b200.meshgraph import SessionMesh
    from nektar_b200.session import read_session
    from tests.session_oracle import oracle_errors, oracle_system
    s = read_session(_REF_PRISM)
    lam = float(s.parameters["Lambda"])
    Ks, b_loc, robin = oracle_system(s, SessionMesh(s))
    assert not robin
    d = _lowenergy_condensed(s, lam, Ks)
    assert {p["shape"] for p in d["parts"]} == {"prism"}
    x, _, _ = _lowenergy_solve(d, b_loc, d["m"].dirichlet_local())
    linf, l2 = oracle_errors(s, d["m"], x)
    printed = lambda v: float("%g" % v)  # noqa: E731  (the demo prints six digits)
    assert abs(printed(l2) - 0.000385246) < 1e-9 and abs(printed(linf) - 0.00539787) < 1e-9
