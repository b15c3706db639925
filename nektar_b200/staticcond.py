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
(nkb_op_create_dense, an HBM-bound batched GEMV); the right-hand side
condensation and the back substitution around it are per-element dense maps
on the device too (nkb_op_create_dense_rect). The element matrices are taken
from the device Helmholtz operators (applied to unit vectors) and condensed
on the host with numpy, as the reference builds its condensed matrices on the
host.

Preconditioners of the condensed system (the reference's Preconditioner
classes for GlobalLinSysIterativeStaticCond):

  "diagonal"   PreconditionerDiagonal: Jacobi on the assembled diag(S).
  "block"      PreconditionerBlock::BlockPreconditionerCG
               (PreconditionerBlock.cpp:123-420): the assembled S restricted
               to each mesh edge's and face's interior modes, inverted; the
               vertex modes keep Jacobi.
  "lowenergy"  PreconditionerLowEnergy (PreconditionerLowEnergy.cpp): the
               boundary space is changed to the low-energy basis of the
               reference element, S~ = R S R^T per element
               (v_TransformedSchurCompl), the CG runs on S~ with the block
               step of "block" built from S~, and the solution is mapped back
               with R^T (v_DoTransformCoeffsFromLowEnergy). Hexahedra,
               tetrahedra and prisms (the prism's transform assembled from the
               hexahedron's and the tetrahedron's). On meshes of variable
               order the transforms are built at the highest order and cut
               down to each element's modes (ExtractLocMat), and the modes a
               lower-order neighbour lacks are masked out of S, the
               right-hand side and the solution (CreateVariablePMask).
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
    """K (nelmt, nc, nc) of an Operator: its application to unit vectors,
    on the device (nkb_op_element_matrices)."""
    import nektar_b200 as nb
    nc, ne = op.in_size // op.nelmt, op.nelmt
    K = np.empty((ne, nc, nc))
    nb.check(nb.lib().nkb_op_element_matrices(op.h, K.ctypes.data, nb.HOST_PTRS, None))
    return K


# vertices of the reference elements the LowEnergy transform is built on
# (PreconditionerLowEnergy::CreateRefHexGeom / CreateRefTetGeom,
# PreconditionerLowEnergy.cpp:1489-1661): the unit cube and the regular
# tetrahedron of edge 2
_S3, _S6 = 3.0 ** 0.5, 6.0 ** 0.5
REFERENCE_VERTICES = {
    "hex": [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1],
            [0, 1, 1]],
    "tet": [[-1, -1 / _S3, -1 / _S6], [1, -1 / _S3, -1 / _S6], [0, 2 / _S3, -1 / _S6],
            [0, 0, 3 / _S6]],
}


def reference_geometry(shape, nm):
    """(T, nq, jac, df) of the reference element at nm modes and nm+1 points
    (GLL, and Gauss-Radau in collapsed directions, as SetUpReferenceElements
    sets up its bases, PreconditionerLowEnergy.cpp:1662-1760)."""
    from . import shape_tables
    from .meshgraph import element_geometry
    if shape not in REFERENCE_VERTICES:
        raise NotImplementedError("low-energy reference element: %s" % shape)
    T, nq = shape_tables(shape, nm, nm + 1)
    X = np.asarray(REFERENCE_VERTICES[shape], dtype=np.float64)[None]
    jac, df, _ = element_geometry(shape, X, tuple(np.asarray(z) for z in T["z"]))
    return T, nq, jac, df


def reference_helmholtz(shape, nm, lam, device=0):
    """Helmholtz matrix L + lam M of the reference element (above). The cube's
    is built on the host from the 1-D mass and stiffness matrices (the map
    from [-1,1] to [0,1] scales them by 1/2 and 2); the tetrahedron's is a
    one-element device operator applied to unit vectors."""
    import nektar_b200 as nb
    if shape == "hex":
        z, w, D = nb.points(nb.GLL, nm + 1)
        b, db = nb.basis(nb.MODIFIED_A, nm, z, D)
        B, dB = np.asarray(b).reshape(nm, nm + 1), np.asarray(db).reshape(nm, nm + 1)
        M = 0.5 * (B * w) @ B.T
        L = 2.0 * (dB * w) @ dB.T
        k3 = lambda a, b, c: np.kron(a, np.kron(b, c))  # noqa: E731  (r, q, p): p fastest
        return lam * k3(M, M, M) + k3(M, M, L) + k3(M, L, M) + k3(L, M, M)
    T, nq, jac, df = reference_geometry(shape, nm)
    op = nb.Operator("helmholtz", shape=shape, nm=nm, nq=nq, nelmt=1, T=T, jac=jac, df=df,
                     deformed=True, device=device)
    try:
        op.set_factors(lam)
        return element_matrices(op)[0]
    finally:
        op.close()


def _entities(shape, nm, bm):
    """Positions (in the boundary-mode order bm) of each vertex, edge and face
    of a shape, and which vertices each edge and face has."""
    verts, edges, faces = topology(shape, nm)
    pos = {int(m): k for k, m in enumerate(bm)}
    V = [pos[m] for m in verts]
    E = [np.array([pos[m] for m, _ in lst], dtype=np.int64) for _, _, lst in edges]
    F = [np.array([pos[m] for m, _, _ in lst], dtype=np.int64) for _, _, lst in faces]
    ev = [(a, b) for a, b, _ in edges]
    adj = {}
    for a, b in ev:
        adj.setdefault(a, set()).add(b)
        adj.setdefault(b, set()).add(a)
    fv = []
    for kind, (o, a, c), _ in faces:
        if kind == "T":
            fv.append({o, a, c})
        else:  # the fourth corner is joined to both ends of the frame's axes
            d = (adj[a] & adj[c]) - {o}
            fv.append({o, a, c} | d)
    return V, E, F, ev, fv


def lowenergy_transform(shape, nm, S):
    """R of Expansion3D::v_BuildTransformationMatrix (Expansion3D.cpp
    :2229-2600) from the reference element's Schur complement S (boundary
    modes in sorted order): unit diagonal; for each vertex v,
    R[v, ef] = -S[v, ef] S[ef, ef]^-1 over the interior modes of its three
    edges and three faces; for each edge e, R[e, f] = -S[e, f] S[f, f]^-1 over
    the interior modes of its two faces."""
    bm, _ = boundary_interior(shape, nm)
    V, E, F, ev, fv = _entities(shape, nm, bm)
    R = np.eye(bm.size)
    for v, pv in enumerate(V):
        cols = np.concatenate([E[e] for e, (a, b) in enumerate(ev) if v in (a, b)] +
                              [F[f] for f in range(len(F)) if v in fv[f]])
        if cols.size:
            R[pv, cols] = -S[pv, cols] @ np.linalg.inv(S[np.ix_(cols, cols)])
    for e, (a, b) in enumerate(ev):
        cols = np.concatenate([F[f] for f in range(len(F)) if a in fv[f] and b in fv[f]])
        if E[e].size and cols.size:
            R[np.ix_(E[e], cols)] = -S[np.ix_(E[e], cols)] @ np.linalg.inv(S[np.ix_(cols, cols)])
    return R


# Correspondence tables of PreconditionerLowEnergy::ReSetTetMaxRMat and
# ReSetPrismMaxRMat (PreconditionerLowEnergy.cpp:2043-2315): which vertex,
# edge and face of the reference hexahedron (or tetrahedron) lends its
# transform entries to which vertex, edge and face of the tetrahedron (or
# prism), in the shapes' standard vertex / edge / face numbering.
_TET_FROM_HEX_VE = ([[0, 0, 0], [1, 1, 1], [2, 2, 2], [4, 5, 6]],   # hex vertex
                    [[0, 3, 4], [0, 1, 5], [1, 2, 6], [4, 5, 6]],   # hex edge
                    [[0, 2, 3], [0, 1, 4], [1, 2, 5], [3, 4, 5]])   # tet edge
_PRISM_FROM_HEX_VE = ([[0, 0, 0], [1, 1, 1], [2, 2, 2], [3, 3, 3], [4, 5, 5], [6, 7, 7]],
                      [[0, 3, 4], [0, 1, 5], [1, 2, 6], [2, 3, 7], [4, 5, 9], [6, 7, 11]],
                      [[0, 3, 4], [0, 1, 5], [1, 2, 6], [2, 3, 7], [4, 5, 8], [6, 7, 8]])
_PRISM_FROM_HEX_VF = ([[0, 0], [1, 1], [4, 5], [2, 2], [3, 3], [6, 7]],   # hex vertex
                      [[0, 4], [0, 2], [4, 2], [0, 2], [0, 4], [2, 4]],   # hex face
                      [[0, 0], [1, 1], [4, 4], [2, 2], [3, 3], [5, 5]],   # prism vertex
                      [[0, 4], [0, 2], [4, 2], [0, 2], [0, 4], [2, 4]])   # prism face
_PRISM_FROM_HEX_EF = ([[0], [1, 1], [2], [3, 3], [4], [5], [6], [7], [9, 11]],   # hex edge
                      [[0], [0, 2], [0], [0, 4], [4], [2], [2], [4], [2, 4]],    # hex face
                      [[0], [1, 1], [2], [3, 3], [4], [5], [6], [7], [8, 8]],    # prism edge
                      [[0], [0, 2], [0], [0, 4], [4], [2], [2], [4], [2, 4]])    # prism face
_PRISM_FROM_TET_VF = ([0, 1, 3, 1, 0, 3], [1] * 6, [0, 1, 4, 2, 3, 5], [1, 1, 1, 3, 3, 3])
_PRISM_FROM_TET_EF = ([0, 3, 4, 0, 4, 3], [1] * 6, [0, 4, 5, 2, 6, 7], [1, 1, 1, 3, 3, 3])


def _maps(shape, nm):
    bm, _ = boundary_interior(shape, nm)
    V, E, F, _, _ = _entities(shape, nm, bm)
    return bm.size, V, E, F


def boundary_keys(shape, nm):
    """Identity of each boundary mode (in boundary_interior's order) that
    does not depend on the order: ("v", vertex), ("e", edge, k) for the
    edge's polynomial index k, ("f", face, a, b) for the face's indices."""
    bm, _ = boundary_interior(shape, nm)
    verts, edges, faces = topology(shape, nm)
    key = {m: ("v", v) for v, m in enumerate(verts)}
    for e, (_, _, lst) in enumerate(edges):
        key.update({m: ("e", e, k) for m, k in lst})
    for f, (_, _, lst) in enumerate(faces):
        key.update({m: ("f", f, a, b) for m, a, b in lst})
    return [key[int(m)] for m in bm]


def transform_of_order(shape, nm, nmax, Rmax):
    """The transform of an element of order nm cut from the one built at the
    mesh's highest order nmax (PreconditionerLowEnergy::ExtractLocMat,
    PreconditionerLowEnergy.cpp:2317-2405): unit diagonal and the
    vertex-edge, vertex-face and edge-face entries of Rmax between the modes
    with the same vertex, edge or face and polynomial indices. Rmax has no
    other off-diagonal entries, so this is the submatrix of Rmax on the
    element's modes."""
    if nm == nmax:
        return Rmax
    pos = {k: i for i, k in enumerate(boundary_keys(shape, nmax))}
    sel = np.array([pos[k] for k in boundary_keys(shape, nm)], dtype=np.int64)
    return Rmax[np.ix_(sel, sel)].copy()


def lowenergy_part_transforms(parts, bsign, lam, device=0, reference=None):
    """Sets each part's "R" (its shape's transform at its order), "Rinv" and
    "mask" ((ne, nb) booleans, False on the local boundary modes of sign 0
    that a lower-order neighbour lacks; None when there are none) from the
    transforms of the mesh's highest order (SetupBlockTransformationMatrix
    and CreateVariablePMask, PreconditionerLowEnergy.cpp:940-1045,
    1255-1275)."""
    nmax = max(p["nm"] for p in parts)
    Rs = lowenergy_transforms({p["shape"] for p in parts}, nmax, lam, device, reference)
    ob = 0
    for p in parts:
        nbm = p["bm"].size
        R = transform_of_order(p["shape"], p["nm"], nmax, Rs[p["shape"]])
        mask = bsign[ob:ob + p["ne"] * nbm].reshape(p["ne"], nbm) != 0
        ob += p["ne"] * nbm
        p["R"], p["Rinv"] = R, np.linalg.inv(R)
        p["mask"] = None if mask.all() else mask


def element_transforms(p):
    """The transform applied to a part's elements: R with the columns of the
    masked modes zeroed, R M_e, so that
    S~ = R M S M R^T (v_TransformedSchurCompl), b~ = R M b
    (v_DoTransformBasisToLowEnergy) and x = M R^T x~
    (v_DoTransformCoeffsFromLowEnergy); one (nb, nb) matrix without a mask,
    else one per element."""
    R, mask = p["R"], p.get("mask")
    if R is None or mask is None:
        return R
    return R[None, :, :] * mask[:, None, :]


def lowenergy_transforms(shapes, nm, lam, device=0, reference=None):
    """R per shape for a mesh with the given shapes at nm modes, as
    SetUpReferenceElements (PreconditionerLowEnergy.cpp:1662-1876) sets them
    up: prisms bring in the hexahedron and the tetrahedron; with a
    hexahedron present the tetrahedron's vertex-edge entries come from the
    hexahedron's (ReSetTetMaxRMat), and the prism's transform is assembled
    from the hexahedron's (quadrilateral faces, vertex-edge) and the
    tetrahedron's (triangular faces) entries (ReSetPrismMaxRMat) instead of
    from a prism reference element. reference(shape, nm, lam) gives the
    reference element's matrix (default reference_helmholtz)."""
    if reference is None:
        reference = lambda sh, n, lm: reference_helmholtz(sh, n, lm, device)  # noqa: E731
    need = set(shapes)
    if "prism" in need:
        need |= {"hex", "tet"}
    Rs = {}
    for shape in ("hex", "tet"):
        if shape in need:
            bm, im = boundary_interior(shape, nm)
            Sr = condense(reference(shape, nm, lam)[None], bm, im)[0][0]
            Rs[shape] = lowenergy_transform(shape, nm, Sr)
    if "hex" in Rs and "tet" in Rs:
        _, Vh, Eh, _ = _maps("hex", nm)
        _, Vt, Et, _ = _maps("tet", nm)
        R = Rs["tet"].copy()
        hv, he, te = _TET_FROM_HEX_VE
        for v in range(4):
            for e in range(3):
                R[Vt[v], Et[te[v][e]]] = Rs["hex"][Vh[hv[v][e]], Eh[he[v][e]]]
        Rs["tet"] = R
    if "prism" in need:
        H, T = Rs["hex"], Rs["tet"]
        _, Vh, Eh, Fh = _maps("hex", nm)
        _, Vt, Et, Ft = _maps("tet", nm)
        nbp, Vp, Ep, Fp = _maps("prism", nm)
        R = np.eye(nbp)
        hv, he, pe = _PRISM_FROM_HEX_VE
        for v in range(6):
            for e in range(3):
                R[Vp[v], Ep[pe[v][e]]] = H[Vh[hv[v][e]], Eh[he[v][e]]]
        hv, hf, pv, pf = _PRISM_FROM_HEX_VF
        for v in range(6):
            for f in range(2):
                R[Vp[pv[v][f]], Fp[pf[v][f]]] = H[Vh[hv[v][f]], Fh[hf[v][f]]]
        he, hf, pe, pf = _PRISM_FROM_HEX_EF
        for e in range(9):
            for f in range(len(he[e])):
                R[np.ix_(Ep[pe[e][f]], Fp[pf[e][f]])] = H[np.ix_(Eh[he[e][f]], Fh[hf[e][f]])]
        tv, tf, pv, pf = _PRISM_FROM_TET_VF
        for v in range(6):
            R[Vp[pv[v]], Fp[pf[v]]] = T[Vt[tv[v]], Ft[tf[v]]]
        te, tf, pe, pf = _PRISM_FROM_TET_EF
        for e in range(6):
            R[np.ix_(Ep[pe[e]], Fp[pf[e]])] = T[np.ix_(Et[te[e]], Ft[tf[e]])]
        Rs["prism"] = R
    return {k: v for k, v in Rs.items() if k in shapes}


def entity_index(parts, bmap, bsign, ndir):
    """The integer side of the entity blocks (PreconditionerBlock::
    BlockPreconditionerCG and the LowEnergy block step gather them,
    PreconditionerLowEnergy.cpp:568-760): every mesh edge and face with more
    than one dof and no Dirichlet dof is one block, its rows its global dofs
    in increasing order; blocks are numbered by size, then by first dof.
    Returns (dofs, contributions): dofs[b] the global dofs of block b and,
    per part, a list of (blocks, elements, rows, signs) arrays with one row
    per contribution of an element to a block (rows: the element's boundary
    rows in the block's row order; signs: the edge / face orientation
    signs), one entry per block size."""
    groups = {}
    ob = 0
    for k, p in enumerate(parts):
        ne, nbm = p["ne"], p["bm"].size
        gb = bmap[ob:ob + ne * nbm].reshape(ne, nbm)
        sb = bsign[ob:ob + ne * nbm].reshape(ne, nbm)
        ob += ne * nbm
        _, E, F, _, _ = _entities(p["shape"], p["nm"], p["bm"])
        for L in E + F:
            if L.size < 2:
                continue
            # on meshes of variable order only the modes of nonzero sign (those
            # of the entity's lowest-order element) form the block
            act = sb[:, L] != 0
            cnt = act.sum(axis=1)
            for n in np.unique(cnt):
                if n < 2:
                    continue
                el = np.flatnonzero(cnt == n)
                er = el[:, None]
                Ln = L[np.argsort(~act[el], axis=1, kind="stable")[:, :n]]
                idx = np.take_along_axis(Ln, np.argsort(gb[er, Ln], axis=1), axis=1)
                G = gb[er, idx]
                dirm = G < ndir
                if (dirm.any(axis=1) != dirm.all(axis=1)).any():
                    raise ValueError("an edge or face has Dirichlet and free dofs")
                keep = ~dirm[:, 0]
                groups.setdefault(int(n), []).append((k, el[keep], G[keep], idx[keep],
                                                      sb[er, idx][keep].astype(np.int8)))
    dofs = []
    contrib = [[] for _ in parts]
    for n in sorted(groups):
        G = np.concatenate([g[2] for g in groups[n]])
        uk, first, inv = np.unique(G[:, 0], return_index=True, return_inverse=True)
        if (G != G[first][inv]).any():
            raise ValueError("entities with a shared first dof differ")
        base = len(dofs)
        dofs.extend(G[first])
        o = 0
        for k, el, Gk, idx, sg in groups[n]:
            contrib[k].append((base + inv[o:o + el.size], el, idx, sg))
            o += el.size
    return dofs, contrib


def entity_blocks(parts, bmap, bsign, ndir):
    """Assembled blocks of the condensed matrices (parts' "S", host) over the
    blocks of entity_index: sign_i sign_j S_e[i, j] summed over the elements
    sharing the entity. Returns [(global dofs, inverse)]; dofs outside every
    block are left to Jacobi."""
    dofs, contrib = entity_index(parts, bmap, bsign, ndir)
    inv = [None] * len(dofs)
    sizes = np.array([d.size for d in dofs])
    for n in np.unique(sizes):
        ids = np.flatnonzero(sizes == n)
        acc = np.zeros((ids.size, n, n))
        for p, entries in zip(parts, contrib):
            for blk, el, idx, sg in entries:
                if idx.shape[1] != n:
                    continue
                sub = p["S"][el[:, None, None], idx[:, :, None], idx[:, None, :]]
                sgd = sg.astype(np.float64)
                np.add.at(acc, blk - ids[0], sub * (sgd[:, :, None] * sgd[:, None, :]))
        for b, Minv in zip(ids, np.linalg.inv(acc)):
            inv[b] = Minv
    return list(zip(dofs, inv))


def _block_layout(dofs, device):
    """bptr of entity_index's blocks and a zeroed device buffer for them
    (n_b * n_b doubles each)."""
    import torch
    sizes = np.array([d.size for d in dofs], dtype=np.int64)
    bptr = np.zeros(len(dofs) + 1, dtype=np.int32)
    bptr[1:] = np.cumsum(sizes)
    A = torch.zeros(int((sizes ** 2).sum()), dtype=torch.float64, device="cuda:%d" % device)
    return bptr, A


def contribution_arrays(entries, nblk):
    """One part's contributions (entity_index) as nkb_blocks_accumulate takes
    them: (cptr, celm, cloc, csgn), contributions grouped by block in a
    stable order."""
    blk = np.concatenate([e[0] for e in entries])
    order = np.argsort(blk, kind="stable")  # contributions grouped by block
    el = np.concatenate([e[1] for e in entries])[order].astype(np.int32)
    # rows and signs of every contribution, padded to the widest block, put
    # in that order and unpadded
    nmax = max(e[2].shape[1] for e in entries)
    rows = np.zeros((blk.size, nmax), dtype=np.int32)
    sgns = np.zeros((blk.size, nmax), dtype=np.int8)
    width = np.zeros(blk.size, dtype=np.int64)
    o = 0
    for b, _, idx, sg in entries:
        rows[o:o + b.size, :idx.shape[1]] = idx
        sgns[o:o + b.size, :idx.shape[1]] = sg
        width[o:o + b.size] = idx.shape[1]
        o += b.size
    used = np.arange(nmax)[None, :] < width[order][:, None]
    cloc = np.ascontiguousarray(rows[order][used])
    csgn = np.ascontiguousarray(sgns[order][used])
    cptr = np.searchsorted(blk[order], np.arange(nblk + 1)).astype(np.int32)
    return cptr, el, cloc, csgn


def _blocks_accumulate(bptr, A, p, S, entries, device):
    """Adds one part's contributions (entity_index) from its condensed
    matrices S (device tensor) to the blocks A (nkb_blocks_accumulate)."""
    import ctypes

    import nektar_b200 as nb
    if not entries:
        return
    nblk = bptr.size - 1
    cptr, el, cloc, csgn = contribution_arrays(entries, nblk)
    ip = ctypes.POINTER(ctypes.c_int)
    nb.check(nb.lib().nkb_blocks_accumulate(
        nblk, bptr.ctypes.data_as(ip), int(el.size), cptr.ctypes.data_as(ip),
        el.ctypes.data_as(ip), cloc.ctypes.data_as(ip),
        csgn.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)), p["ne"], p["bm"].size,
        ctypes.c_void_p(S.data_ptr()), ctypes.c_void_p(A.data_ptr()), device, None))


def _blocks_invert(bptr, A, device):
    import ctypes

    import nektar_b200 as nb
    nb.check(nb.lib().nkb_blocks_invert(bptr.size - 1,
                                        bptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        ctypes.c_void_p(A.data_ptr()), device, None))


def _mask_groups(p):
    """[(element rows or None for all, transform)]: the part's elements
    grouped by their variable-order mask, one transform per group."""
    if p.get("mask") is None:
        return [(None, p["R"])]
    pats, inv = np.unique(p["mask"], axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    return [(np.flatnonzero(inv == g), p["R"] * pat[None, :]) for g, pat in enumerate(pats)]


def _condense_device(op, p, device):
    """(S, W, V) of an Operator's elements as device tensors: its element
    matrices built on the device and condensed there (nkb_condense), one
    call per group of elements that share a transform."""
    import ctypes

    import torch

    import nektar_b200 as nb
    bm, im = p["bm"], p["im"]
    nc, ne = op.in_size // op.nelmt, op.nelmt
    nbm, ni = len(bm), len(im)
    dev = "cuda:%d" % device
    K = torch.empty((ne, nc, nc), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    nb.check(nb.lib().nkb_op_element_matrices(op.h, ctypes.c_void_p(K.data_ptr()),
                                              nb.DEVICE_PTRS, None))
    S = torch.empty((ne, nbm, nbm), dtype=torch.float64, device=dev)
    W = torch.empty((ne, nbm, nc), dtype=torch.float64, device=dev)
    V = torch.empty((ne, nc, nbm + ni), dtype=torch.float64, device=dev)
    bmi = np.ascontiguousarray(bm, dtype=np.int32)
    imi = np.ascontiguousarray(im, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    for rows, R in _mask_groups(p):
        if rows is None:
            Kg, Sg, Wg, Vg = K, S, W, V
        else:
            ri = torch.as_tensor(rows, device=dev)
            Kg = K.index_select(0, ri)
            Sg, Wg, Vg = (torch.empty((rows.size,) + t.shape[1:], dtype=torch.float64, device=dev)
                          for t in (S, W, V))
        Rc = None if R is None else np.ascontiguousarray(R, dtype=np.float64)
        nb.check(nb.lib().nkb_condense(int(Kg.shape[0]), nc, ctypes.c_void_p(Kg.data_ptr()), nbm,
                                       bmi.ctypes.data_as(ip), ni, imi.ctypes.data_as(ip),
                                       None if Rc is None else Rc.ctypes.data_as(
                                           ctypes.POINTER(ctypes.c_double)),
                                       ctypes.c_void_p(Sg.data_ptr()),
                                       ctypes.c_void_p(Wg.data_ptr()),
                                       ctypes.c_void_p(Vg.data_ptr()), device, None))
        if rows is not None:
            torch.cuda.synchronize(dev)
            S[ri], W[ri], V[ri] = Sg, Wg, Vg
            del Kg, Sg, Wg, Vg
    torch.cuda.synchronize(dev)
    del K
    return S, W, V


def condense(K, bm, im):
    """(S, C, Kii_inv, Kib) of element matrices: S = Kbb - C Kib, C = Kbi Kii^-1."""
    Kbb = K[:, bm[:, None], bm]
    Kbi = K[:, bm[:, None], im]
    Kib = K[:, im[:, None], bm]
    Kii_inv = np.linalg.inv(K[:, im[:, None], im])
    C = Kbi @ Kii_inv
    return Kbb - C @ Kib, C, Kii_inv, Kib


def solve_maps(C, Kii_inv, Kib, bm, im, R=None):
    """Per-element matrices of the two steps around the condensed CG
    (GlobalLinSysStaticCond::v_Solve, GlobalLinSysStaticCond.cpp:98-227):

      W (nb x nc):        b~ = R (b_b - C b_i)          from the local b_e
      V (nc x (nb + ni)): x_b = R^T x~,
                          x_i = Kii^-1 b_i - Kii^-1 Kib R^T x~
                                                        from [x~_e, b_i,e]

    with R the low-energy transform (identity if None; one for all elements
    or one per element); V's rows are in the element's local mode order."""
    ne, nbm, ni = C.shape
    nc = nbm + ni
    R = np.eye(nbm) if R is None else R
    RT = np.swapaxes(R, -1, -2)
    W = np.zeros((ne, nbm, nc))
    W[:, :, bm] = R
    W[:, :, im] = -(R @ C)
    V = np.zeros((ne, nc, nbm + ni))
    V[:, bm, :nbm] = RT
    V[:, im, :nbm] = -(Kii_inv @ (Kib @ RT))
    V[:, im, nbm:] = Kii_inv
    return W, V


def condensed_parts(collections):
    """One dict per collection (shape, nm, number of elements) with its
    boundary / interior mode split and its offset in the local space."""
    parts, off = [], 0
    for shape, nm, ne in collections:
        nc = ncoeffs(shape, nm)
        bm, im = boundary_interior(shape, nm)
        parts.append(dict(nc=nc, ne=ne, bm=bm, im=im, off=off, shape=shape, nm=nm, R=None,
                          mask=None))
        off += ne * nc
    return parts


def boundary_map(parts, gmap, sign, nglob, ndir):
    """(bmap, bsign, number of boundary dofs): the local boundary modes' map
    to the boundary dofs, renumbered in their original order (the Dirichlet
    dofs first, as they were), and their signs."""
    gmap = np.asarray(gmap)
    sign = np.ones(gmap.size) if sign is None else np.asarray(sign, dtype=np.float64)
    bglob, bsign = [], []
    for p in parts:
        ne, nc, off = p["ne"], p["nc"], p["off"]
        bglob.append(gmap[off:off + ne * nc].reshape(ne, nc)[:, p["bm"]].ravel())
        bsign.append(sign[off:off + ne * nc].reshape(ne, nc)[:, p["bm"]].ravel())
    bglob = np.concatenate(bglob)
    ids = np.unique(bglob)
    if ndir and (ids[:ndir] != np.arange(ndir)).any():
        raise ValueError("Dirichlet dofs must be boundary dofs numbered first")
    renum = np.full(nglob, -1, dtype=np.int64)
    renum[ids] = np.arange(ids.size)
    return renum[bglob].astype(np.int32), np.concatenate(bsign), int(ids.size)


class StaticCondSys:
    """Statically condensed Helmholtz system over Helmholtz collection
    operators (Operator) with the C0 map of the full local space. A solve is
    three device steps: the right-hand side condensation (per-element dense
    W), the CG on the condensed system, and the interior back substitution
    (per-element dense V).

    The set-up (element matrices, condensation, the maps W and V) runs on the
    device (setup="device": nkb_op_element_matrices into device memory, then
    nkb_condense, the batched Cholesky condensation) or on the host
    (setup="host": numpy, or when the element matrices are given); the
    low-energy transform of a reference element and the block inverses of
    the Block / LowEnergy preconditioners are built on the host."""

    def __init__(self, ops, gmap, nglob, ndir, sign=None, device=0, matrices=None,
                 precon="diagonal", lam=None, setup="device"):
        """precon: "diagonal", "block" or "lowenergy"; lam: the operators'
        Helmholtz lambda, which the low-energy reference element uses
        (default: the one last given to the operators' set_factors)."""
        import nektar_b200 as nb
        if precon not in ("diagonal", "block", "lowenergy"):
            raise ValueError("precon %r" % (precon,))
        if setup not in ("device", "host"):
            raise ValueError("setup %r" % (setup,))
        t0 = time.perf_counter()
        self.ops = list(ops)
        self.precon = precon
        self.setup = "host" if matrices is not None else setup
        # wall seconds of the set-up's phases
        self.setup_breakdown = {}
        tp = [t0]

        def phase(name):
            t = time.perf_counter()
            self.setup_breakdown[name] = self.setup_breakdown.get(name, 0.0) + t - tp[0]
            tp[0] = t
        self.parts = condensed_parts([(op.shape, op.nm, op.nelmt) for op in self.ops])
        self.nloc = sum(p["ne"] * p["nc"] for p in self.parts)
        self.bmap, self.bsign, self.nglob_b = boundary_map(self.parts, gmap, sign, nglob, ndir)
        self.ndir, self.nglob = int(ndir), int(nglob)
        phase("maps")
        if precon == "lowenergy":
            if lam is None:
                lam = getattr(self.ops[0], "lam", None)
            if lam is None:
                raise ValueError("lowenergy needs the Helmholtz lambda")
            lowenergy_part_transforms(self.parts, self.bsign, float(lam), device)
            phase("lowenergy_transform")
        need_blocks = precon != "diagonal"
        need_host_S = need_blocks and self.setup == "host"
        if need_blocks and self.setup == "device":
            dofs, contrib = entity_index(self.parts, self.bmap, self.bsign, self.ndir)
            bptr, A = _block_layout(dofs, device)
            phase("blocks")
        self.dense, self.W, self.V = [], [], []
        for k, (op, p) in enumerate(zip(self.ops, self.parts)):
            if self.setup == "device":
                S, W, V = _condense_device(op, p, device)
                phase("condense")
                if need_blocks:
                    _blocks_accumulate(bptr, A, p, S, contrib[k], device)
                    phase("blocks")
                self.W.append(nb.DenseOperator.from_device(W, device=device))
                self.V.append(nb.DenseOperator.from_device(V, device=device))
                self.dense.append(nb.DenseOperator.from_device(S, device=device))
                del S, W, V
                phase("dense_operators")
                continue
            K = element_matrices(op) if matrices is None else matrices[k]
            S, C, Kii_inv, Kib = condense(K, p["bm"], p["im"])
            del K
            Re = element_transforms(p)
            if Re is not None:
                S = Re @ S @ np.swapaxes(Re, -1, -2)  # v_TransformedSchurCompl
            W, V = solve_maps(C, Kii_inv, Kib, p["bm"], p["im"], Re)
            del C, Kii_inv, Kib
            self.W.append(nb.DenseOperator(W, device=device))
            del W
            self.V.append(nb.DenseOperator(V, device=device))
            del V
            if need_host_S:
                p["S"] = S
            self.dense.append(nb.DenseOperator(S, device=device))
            del S
            phase("condense")
        blocks = None
        if need_host_S:
            blocks = entity_blocks(self.parts, self.bmap, self.bsign, self.ndir)
            self.nblocks = len(blocks)
        elif need_blocks:
            if dofs:
                _blocks_invert(bptr, A, device)
            self.nblocks = len(dofs)
        else:
            self.nblocks = 0
        for p in self.parts:
            p.pop("S", None)
        phase("blocks")
        self.sys = nb.GlobalLinSys(self.dense, self.bmap, self.nglob_b, self.ndir,
                                   sign=self.bsign, device=device)
        if blocks:
            self.sys.set_blocks(blocks)
        elif need_blocks and self.nblocks:
            self.sys.set_block_inverses(bptr, np.concatenate(dofs), A.data_ptr())
            del A
        phase("linsys")
        self.setup_s = time.perf_counter() - t0

    def _parts_of(self, v):
        for p in self.parts:
            yield p, v[p["off"]:p["off"] + p["ne"] * p["nc"]].reshape(p["ne"], p["nc"])

    def condense_rhs(self, b_loc):
        """Condensed (and, for lowenergy, transformed) boundary right-hand
        side, element by element (device)."""
        b = np.asarray(b_loc, dtype=np.float64)
        return np.concatenate([W(be.ravel()) for W, (_, be) in zip(self.W, self._parts_of(b))])

    def solve(self, b_loc, x_loc=None, tol=1e-9, maxit=5000, check_interval=16,
              raise_on_maxit=True):
        """Local rhs and local Dirichlet values -> local solution, report
        (the report's iterations and device time are the condensed CG's)."""
        b = np.asarray(b_loc, dtype=np.float64)
        xb0 = []
        if x_loc is None:
            xb0 = np.zeros(self.bmap.size)
        else:
            for p, xe in self._parts_of(np.asarray(x_loc, dtype=np.float64)):
                xe = xe[:, p["bm"]]
                if p["R"] is not None:
                    # v_CoeffsFwdTransform of the whole local boundary vector
                    # (R^-T x, GlobalLinSysStaticCond.cpp:166-172): the lifting
                    # then equals R (b - S x) and the result x + R^T (G d~), so
                    # local Dirichlet values that differ between elements (the
                    # reference's boundary projection allows that) never
                    # reach the free modes
                    xe = xe @ p["Rinv"]
                xb0.append(xe.ravel())
            xb0 = np.concatenate(xb0)
        xb, rep = self.sys.solve(self.condense_rhs(b), xb0, tol=tol, maxit=maxit,
                                 check_interval=check_interval, raise_on_maxit=raise_on_maxit)
        x = np.empty(self.nloc)
        ob = 0
        for V, (p, be) in zip(self.V, self._parts_of(b)):
            ne, nbm = p["ne"], p["bm"].size
            z = np.concatenate([xb[ob:ob + ne * nbm].reshape(ne, nbm), be[:, p["im"]]], axis=1)
            x[p["off"]:p["off"] + ne * p["nc"]] = V(z.ravel())
            ob += ne * nbm
        return x, rep

    def close(self):
        self.sys.close()
        for d in self.dense + self.W + self.V:
            d.close()
