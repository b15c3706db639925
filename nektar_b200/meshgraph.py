"""Mesh graph of a session for the B200 path: element frames, geometric
factors at the quadrature points, the C0 local -> global map with Dirichlet
degrees of freedom first, and the Dirichlet values, for meshes of
hexahedra, prisms and tetrahedra (one operator collection per shape and
order, as the reference groups them).

Element frames follow the reference's geometry classes: the element lists
its faces in a fixed order, local edges are the faces' shared edges, local
vertices follow the edge chain (HexGeom::SetUpLocalEdges / Vertices,
SpatialDomains/HexGeom.cpp:200-430; PrismGeom.cpp:185-391; TetGeom.cpp:
113-308). Standard-region vertices:

    hex    v0..v3 = (-1,-1,-1) (1,-1,-1) (1,1,-1) (-1,1,-1), v4..v7 the same at +1
    prism  v0..v3 as the hex, v4 = (-1,-1,1), v5 = (-1,1,1)
    tet    v0 = (-1,-1,-1), v1 = (1,-1,-1), v2 = (-1,1,-1), v3 = (-1,-1,1)

Geometry: straight-sided maps, linear in the vertex coordinates through
the vertex shape functions (the two-mode coordinate expansion), evaluated at
the collapsed quadrature points mapped to the standard region; jac = det
dx/dxi and df[k*3+j] = d xi_j / d x_k in the Collections layout (GeomFactors
.cpp:248-477).

Continuity (AssemblyMapCG, AssemblyMapCG.cpp:1322-2300): each shape's modes
are split into vertex, edge, face and interior modes by the reference's maps
(StdHexExp / StdPrismExp / StdTetExp GetVertexMap,
GetEdgeInteriorToElementMap, GetTraceInteriorToElementMap; e.g.
StdTetExp.cpp:1075-1700, StdPrismExp.cpp:942-1760). Edge modes are numbered
along the edge from its lower to its higher global vertex id; mode k of an
element edge running the other way gets (-1)^k. Quadrilateral face modes
(a, b) are numbered in a frame anchored at the face's lowest global vertex,
first axis towards the lower of its neighbours; an element's face frame maps
to it by a transposition and reflections (sign (-1)^(a s_a + b s_b)).
Triangular faces have only two admissible relative orientations (the
collapsed apex shared, the other axis possibly reflected): modes are numbered
from the lower of the two base vertices, and a reflected element face gets
(-1)^a; a mesh whose neighbouring triangles disagree on the apex is
rejected, as the reference requires compatible collapsed directions.

Dirichlet values (ExpList::FwdTransBndConstrained on the boundary faces,
QuadExp.cpp:67-170, TriExp::v_FwdTransBndConstrained, SegExp.cpp:81-180):
vertex modes take the point values, edge bubbles the constrained L2
projection at GLL points along the edge, face bubbles the constrained L2
projection with the face's quadrature (GLL x GLL, or GLL x Gauss-Radau on a
triangle) and surface Jacobian. A triangle works in its own frame and
interpolates the data of its edges 1 and 2 from the Gauss-Radau points to
GLL points first, so its apex value is an extrapolation. The local Dirichlet
vector a solve takes is built as the reference builds it
(dirichlet_local): face by face into each face's element, later faces
overwriting, then copied to elements that only touch the boundary; with it
the reference's Hex, Prism and Tet regression errors are reproduced.
"""
import numpy as np

from . import shape_tables
from .session import SessionError

# ---------------------------------------------------------------------------
# standard-region vertices, vertex shape functions, collapsed -> standard
# ---------------------------------------------------------------------------
STD_VERTS = {
    "hex": np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64),
    "prism": np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                       [-1, -1, 1], [-1, 1, 1]], dtype=np.float64),
    "tet": np.array([[-1, -1, -1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float64),
}
NVERTS = {"hex": 8, "prism": 6, "tet": 4}
NFACES = {"hex": 6, "prism": 5, "tet": 4}
FACE_KINDS = {"hex": "QQQQQQ", "prism": "QTQTQ", "tet": "TTTT"}


def shape_functions(shape, xi):
    """N (npts, nv) and dN/dxi (npts, nv, 3) of the straight-sided map."""
    x1, x2, x3 = xi[:, 0], xi[:, 1], xi[:, 2]
    h = lambda v: 0.5 * (1.0 + v)  # noqa: E731
    m = lambda v: 0.5 * (1.0 - v)  # noqa: E731
    n = xi.shape[0]
    if shape == "hex":
        s = STD_VERTS["hex"]
        fac = 0.5 * (1.0 + xi[:, None, :] * s[None, :, :])
        N = fac.prod(axis=2)
        dN = np.empty((n, 8, 3))
        for j in range(3):
            d = fac.copy()
            d[:, :, j] = 0.5 * s[None, :, j]
            dN[:, :, j] = d.prod(axis=2)
        return N, dN
    if shape == "prism":
        la, lb, lc = -0.5 * (x1 + x3), h(x1), h(x3)
        m0, m1 = m(x2), h(x2)
        N = np.stack([la * m0, lb * m0, lb * m1, la * m1, lc * m0, lc * m1], axis=1)
        dla = np.array([-0.5, 0.0, -0.5])
        dlb = np.array([0.5, 0.0, 0.0])
        dlc = np.array([0.0, 0.0, 0.5])
        dm0 = np.array([0.0, -0.5, 0.0])
        dm1 = np.array([0.0, 0.5, 0.0])
        dN = np.empty((n, 6, 3))
        for v, (l, dl, mm, dmm) in enumerate(((la, dla, m0, dm0), (lb, dlb, m0, dm0),
                                               (lb, dlb, m1, dm1), (la, dla, m1, dm1),
                                               (lc, dlc, m0, dm0), (lc, dlc, m1, dm1))):
            dN[:, v, :] = dl[None, :] * mm[:, None] + l[:, None] * dmm[None, :]
        return N, dN
    if shape == "tet":
        N = np.stack([-0.5 * (1.0 + x1 + x2 + x3), h(x1), h(x2), h(x3)], axis=1)
        dN = np.broadcast_to(np.array([[-0.5, -0.5, -0.5], [0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5]]),
                             (n, 4, 3)).copy()
        return N, dN
    raise SessionError("unsupported shape %r" % shape)


def collapsed_to_standard(shape, e1, e2, e3):
    """Standard-region coordinates of collapsed coordinates (the Duffy maps
    of StdPrismExp / StdTetExp)."""
    if shape == "hex":
        return e1, e2, e3
    if shape == "prism":
        return 0.5 * (1 + e1) * (1 - e3) - 1, e2, e3
    return 0.25 * (1 + e1) * (1 - e2) * (1 - e3) - 1, 0.5 * (1 + e2) * (1 - e3) - 1, e3


def edge_bubble(shape, a, b, xi):
    """The quadratic edge mode of local edge (a, b) of a shape (the modified
    basis's mode 2 on that edge, zero on the other edges and faces not
    holding it) and its gradient at standard points xi (n, 3): the product
    of the edge's two end barycentrics (tet; prism edges in a triangle,
    times the extrusion factor), or (1 - t^2)/4 along the edge times the
    linear factors across it (hexahedra, prism edges along the extrusion)."""
    V = STD_VERTS[shape]
    n = xi.shape[0]
    one = np.ones(n)
    if shape == "hex":
        d = int(np.nonzero(V[a] != V[b])[0][0])
        fac, grad = [], []
        for ax in range(3):
            t = xi[:, ax]
            if ax == d:
                fac.append(0.25 * (1 - t * t))
                grad.append(-0.5 * t)
            else:
                sg = V[a][ax]
                fac.append(0.5 * (1 + sg * t))
                grad.append(0.5 * sg * one)
        phi = fac[0] * fac[1] * fac[2]
        dphi = np.stack([grad[0] * fac[1] * fac[2], fac[0] * grad[1] * fac[2],
                         fac[0] * fac[1] * grad[2]], axis=1)
        return phi, dphi
    x1, x2, x3 = xi[:, 0], xi[:, 1], xi[:, 2]
    if shape == "tet":
        lam = [-0.5 * (1 + x1 + x2 + x3), 0.5 * (1 + x1), 0.5 * (1 + x2), 0.5 * (1 + x3)]
        dl = [np.array([-0.5, -0.5, -0.5]), np.array([0.5, 0, 0]), np.array([0, 0.5, 0]),
              np.array([0, 0, 0.5])]
        return lam[a] * lam[b], lam[a][:, None] * dl[b] + lam[b][:, None] * dl[a]
    # prism: triangle (xi1, xi3) barycentrics, extrusion along xi2
    lam = [-0.5 * (x1 + x3), 0.5 * (1 + x1), 0.5 * (1 + x3)]
    dl = [np.array([-0.5, 0, -0.5]), np.array([0.5, 0, 0]), np.array([0, 0, 0.5])]
    tri = {(-1, -1): 0, (1, -1): 1, (-1, 1): 2}
    ta, tb = tri[(V[a][0], V[a][2])], tri[(V[b][0], V[b][2])]
    if ta != tb:  # an edge of a triangle, at xi2 = +-1
        sg = V[a][1]
        h, dh = 0.5 * (1 + sg * x2), np.array([0, 0.5 * sg, 0])
        phi = lam[ta] * lam[tb] * h
        dphi = (lam[ta][:, None] * dl[tb] + lam[tb][:, None] * dl[ta]) * h[:, None] + \
            (lam[ta] * lam[tb])[:, None] * dh
        return phi, dphi
    b2 = 0.25 * (1 - x2 * x2)
    return lam[ta] * b2, dl[ta][None, :] * b2[:, None] + \
        (lam[ta] * (-0.5 * x2))[:, None] * np.array([0, 1.0, 0])


def face_bubble_coeff(pts):
    """The (2, 2) mode coefficient (3,) of a quadrilateral face's quadratic
    curve, its 3 x 3 points in tensor order (QuadGeom::v_FillGeom projects
    the interpolant of the points on the face's modes; the biquadratic's
    (2, 2) coefficient is 16 (centre - mean of the midpoints x 2 + mean of
    the corners), the same for every orientation and either point order)."""
    p = np.asarray(pts, dtype=np.float64)
    return 16.0 * (p[4] - 0.5 * (p[1] + p[3] + p[5] + p[7]) + 0.25 * (p[0] + p[2] + p[6] + p[8]))


def face_bubble(shape, lf, xi):
    """The (2, 2) mode of local quadrilateral face lf of a hexahedron or
    prism and its gradient at standard points xi (n, 3): the two in-face
    quadratic bubbles (1 - t^2)/4 times the linear factor across the face
    (hexahedra); for a prism the product of the face's two triangle
    barycentrics (its (2, *) collapsed modes) times (1 - xi2^2)/4. On the
    face it is the face's own (2, 2) mode, so the coefficient of the face
    carries over unchanged (HexGeom / PrismGeom::v_FillGeom)."""
    V = STD_VERTS[shape]
    _, _, faces = topology(shape, 3)
    kind, frame, _ = faces[lf]
    if kind != "Q":
        raise ValueError("face %d of a %s is a triangle" % (lf, shape))
    n = xi.shape[0]
    one = np.ones(n)
    if shape == "hex":
        o, a, c = (V[v] for v in frame)
        ax = int(np.nonzero((o == a) & (o == c))[0][0])
        fac, grad = [], []
        for d in range(3):
            t = xi[:, d]
            if d == ax:
                fac.append(0.5 * (1 + o[d] * t))
                grad.append(0.5 * o[d] * one)
            else:
                fac.append(0.25 * (1 - t * t))
                grad.append(-0.5 * t)
        phi = fac[0] * fac[1] * fac[2]
        dphi = np.stack([grad[0] * fac[1] * fac[2], fac[0] * grad[1] * fac[2],
                         fac[0] * fac[1] * grad[2]], axis=1)
        return phi, dphi
    if shape != "prism":
        raise ValueError("no quadrilateral faces on a %s" % shape)
    x1, x2, x3 = xi[:, 0], xi[:, 1], xi[:, 2]
    lam = [-0.5 * (x1 + x3), 0.5 * (1 + x1), 0.5 * (1 + x3)]
    dl = [np.array([-0.5, 0, -0.5]), np.array([0.5, 0, 0]), np.array([0, 0, 0.5])]
    tri = {(-1, -1): 0, (1, -1): 1, (-1, 1): 2}
    ta, tb = sorted({tri[(V[v][0], V[v][2])] for v in frame})
    b2, db2 = 0.25 * (1 - x2 * x2), -0.5 * x2
    phi = lam[ta] * lam[tb] * b2
    dphi = (lam[ta][:, None] * dl[tb] + lam[tb][:, None] * dl[ta]) * b2[:, None] + \
        (lam[ta] * lam[tb] * db2)[:, None] * np.array([0, 1.0, 0])
    return phi, dphi


def element_geometry(shape, X, z, curves=None, faces=None):
    """jac (nelmt*nt,), df (9, nelmt*nt), coordinates (3, nelmt*nt) of
    elements with vertex coordinates X (nelmt, nv, 3) at the collapsed tensor
    points z = (z0, z1, z2) (point q = (k nq1 + j) nq0 + i). curves: per
    element a list of (local edge (a, b), mode-2 coefficient c (3,)) of its
    quadratic curved edges; faces: per element a list of (local face,
    (2, 2) coefficient (3,)) of its curved quadrilateral faces; both added to
    the vertex map as the reference's geometry expansions add the edges' and
    faces' coefficients (Geometry3D::v_FillGeom; the factors are the map's
    exact derivatives at the points)."""
    e1, e2, e3 = np.meshgrid(z[0], z[1], z[2], indexing="ij")  # [i, j, k]
    e = [a.transpose(2, 1, 0).reshape(-1) for a in (e1, e2, e3)]
    xi = np.stack(collapsed_to_standard(shape, *e), axis=1)
    N, dN = shape_functions(shape, xi)
    x = np.einsum("pc,ecd->edp", N, X)
    J = np.einsum("pcj,ecd->epdj", dN, X)  # J[e, p, d, j] = d x_d / d xi_j
    for el, lst in enumerate(curves or []):
        for (a, b), c in lst:
            phi, dphi = edge_bubble(shape, a, b, xi)
            x[el] += np.asarray(c)[:, None] * phi[None, :]
            J[el] += np.asarray(c)[None, :, None] * dphi[:, None, :]
    for el, lst in enumerate(faces or []):
        for lf, c in lst:
            phi, dphi = face_bubble(shape, lf, xi)
            x[el] += np.asarray(c)[:, None] * phi[None, :]
            J[el] += np.asarray(c)[None, :, None] * dphi[:, None, :]
    det = np.linalg.det(J)
    if np.any(det <= 0):
        raise SessionError("element with a non-positive Jacobian")
    inv = np.linalg.inv(J)  # d xi_j / d x_k at [e, p, j, k]
    ne, nt = X.shape[0], xi.shape[0]
    df = np.empty((9, ne * nt))
    for k in range(3):
        for j in range(3):
            df[k * 3 + j] = inv[:, :, j, k].reshape(-1)
    return det.reshape(-1), df, x.transpose(1, 0, 2).reshape(3, -1)


def hex_geometry(X, z):
    """element_geometry for hexahedra at the same points in every direction."""
    return element_geometry("hex", X, (z, z, z))


# ---------------------------------------------------------------------------
# local frames (reference geometry classes)
# ---------------------------------------------------------------------------

def _shared_edge(fa, fb, faces, what):
    common = [e for e in faces[fa][1] if e in faces[fb][1]]
    if len(common) != 1:
        raise SessionError("faces %d and %d share %d edges (%s)" % (fa, fb, len(common), what))
    return common[0]


def _chain(E, first, second, nxt, eid):
    a, b = E[first]
    if a in E[second]:
        v = [b, a]
    elif b in E[second]:
        v = [a, b]
    else:
        raise SessionError("edges of element %d do not connect" % eid)
    for k in nxt:
        x, y = E[k]
        if x == v[-1]:
            v.append(y)
        elif y == v[-1]:
            v.append(x)
        else:
            raise SessionError("edges of element %d do not connect" % eid)
    return v


def _other_end(edge, v, eid):
    a, b = edge
    if a == v:
        return b
    if b == v:
        return a
    raise SessionError("edges of element %d do not connect" % eid)


def local_vertices(geom, eid):
    """Global vertex ids of element eid in its local order."""
    shape, F = geom.elements[eid]
    faces = geom.faces
    if len(F) != NFACES[shape]:
        raise SessionError("element %d has %d faces" % (eid, len(F)))
    for f, kind in zip(F, FACE_KINDS[shape]):
        if faces[f][0] != kind:
            raise SessionError("face %d of %s %d is not a %s" % (f, shape, eid,
                               "quadrilateral" if kind == "Q" else "triangle"))
    if shape == "hex":  # HexGeom.cpp:200-430
        e = [None] * 12
        for f in range(1, 5):
            e[f - 1] = _shared_edge(F[0], F[f], faces, "bottom")
        e[4] = _shared_edge(F[1], F[4], faces, "vertical")
        for f in range(1, 4):
            e[f + 4] = _shared_edge(F[f], F[f + 1], faces, "vertical")
        for f in range(1, 5):
            e[f + 7] = _shared_edge(F[5], F[f], faces, "top")
        E = [geom.edges[k] for k in e]
        return _chain(E, 0, 1, (1, 2), eid) + _chain(E, 8, 9, (9, 10), eid)
    if shape == "prism":  # PrismGeom.cpp:185-391
        e = [None] * 9
        for f in range(1, 5):
            e[f - 1] = _shared_edge(F[0], F[f], faces, "bottom")
        e[4] = _shared_edge(F[1], F[4], faces, "vertical")
        for f in range(1, 4):
            e[f + 4] = _shared_edge(F[f], F[f + 1], faces, "vertical")
        e[8] = _shared_edge(F[2], F[4], faces, "top")
        E = [geom.edges[k] for k in e]
        v = _chain(E, 0, 1, (1, 2), eid)
        a, b = E[8]
        if a in E[4]:
            v += [a, b]
        elif b in E[4]:
            v += [b, a]
        else:
            raise SessionError("edges of element %d do not connect" % eid)
        return v
    # tet, TetGeom.cpp:113-308
    e = [None] * 6
    for f in range(1, 4):
        e[f - 1] = _shared_edge(F[0], F[f], faces, "bottom")
    e[3] = _shared_edge(F[1], F[3], faces, "vertical")
    e[4] = _shared_edge(F[1], F[2], faces, "vertical")
    e[5] = _shared_edge(F[2], F[3], faces, "vertical")
    E = [geom.edges[k] for k in e]
    v = _chain(E, 0, 1, (1,), eid)
    v.append(_other_end(E[3], v[0], eid))
    return v


def hex_local_vertices(geom, eid):
    return local_vertices(geom, eid)


# ---------------------------------------------------------------------------
# mode maps
# ---------------------------------------------------------------------------

def mode_index(shape, nm):
    """(p, q, r) -> local coefficient index (StdHexExp ordering p fastest;
    StdPrismExp::GetMode, StdPrismExp.cpp:1947-1956; StdTetExp::GetMode,
    StdTetExp.cpp:1864-1893)."""
    if shape == "hex":
        return lambda p, q, r: p + nm * (q + nm * r)
    if shape == "prism":
        Q = R = nm - 1
        return lambda p, q, r: r + q * (R + 1 - p) + (Q + 1) * (p * R + 1 - (p - 2) * (p - 1) // 2)

    def tet(I, J, K):
        cnt = 0
        for i in range(I):
            cnt += (nm - i) * (nm - i + 1) // 2
        for j in range(J):
            cnt += nm - I - j
        return cnt + K
    return tet


def topology(shape, nm):
    """Vertex modes, edges (start, end, [(mode, k)]) and faces (kind, frame,
    [(mode, a, b)]) of a shape at nm modes per direction. Quadrilateral frames
    are (origin, end of axis a, end of axis b); triangular frames (origin, end
    of axis a, apex)."""
    G = mode_index(shape, nm)
    K = range(2, nm)
    if shape == "hex":
        verts = [G(0, 0, 0), G(1, 0, 0), G(1, 1, 0), G(0, 1, 0), G(0, 0, 1), G(1, 0, 1),
                 G(1, 1, 1), G(0, 1, 1)]
        edges = [(0, 1, [(G(k, 0, 0), k) for k in K]), (1, 2, [(G(1, k, 0), k) for k in K]),
                 (3, 2, [(G(k, 1, 0), k) for k in K]), (0, 3, [(G(0, k, 0), k) for k in K]),
                 (0, 4, [(G(0, 0, k), k) for k in K]), (1, 5, [(G(1, 0, k), k) for k in K]),
                 (2, 6, [(G(1, 1, k), k) for k in K]), (3, 7, [(G(0, 1, k), k) for k in K]),
                 (4, 5, [(G(k, 0, 1), k) for k in K]), (5, 6, [(G(1, k, 1), k) for k in K]),
                 (7, 6, [(G(k, 1, 1), k) for k in K]), (4, 7, [(G(0, k, 1), k) for k in K])]
        faces = [("Q", (0, 1, 3), [(G(a, b, 0), a, b) for b in K for a in K]),
                 ("Q", (0, 1, 4), [(G(a, 0, b), a, b) for b in K for a in K]),
                 ("Q", (1, 2, 5), [(G(1, a, b), a, b) for b in K for a in K]),
                 ("Q", (3, 2, 7), [(G(a, 1, b), a, b) for b in K for a in K]),
                 ("Q", (0, 3, 4), [(G(0, a, b), a, b) for b in K for a in K]),
                 ("Q", (4, 5, 7), [(G(a, b, 1), a, b) for b in K for a in K])]
    elif shape == "prism":  # StdPrismExp.cpp:942-1760
        verts = [G(0, 0, 0), G(1, 0, 0), G(1, 1, 0), G(0, 1, 0), G(0, 0, 1), G(0, 1, 1)]
        edges = [(0, 1, [(G(k, 0, 0), k) for k in K]), (1, 2, [(G(1, k, 0), k) for k in K]),
                 (3, 2, [(G(k, 1, 0), k) for k in K]), (0, 3, [(G(0, k, 0), k) for k in K]),
                 (0, 4, [(G(0, 0, k), k) for k in K]), (1, 4, [(G(1, 0, k - 1), k) for k in K]),
                 (2, 5, [(G(1, 1, k - 1), k) for k in K]), (3, 5, [(G(0, 1, k), k) for k in K]),
                 (4, 5, [(G(0, k, 1), k) for k in K])]
        tri = lambda q: [(G(a, q, b), a, b) for a in K for b in range(1, nm - a)]  # noqa: E731
        faces = [("Q", (0, 1, 3), [(G(a, b, 0), a, b) for b in K for a in K]),
                 ("T", (0, 1, 4), tri(0)),
                 ("Q", (1, 2, 4), [(G(1, a, b - 1), a, b) for b in K for a in K]),
                 ("T", (3, 2, 5), tri(1)),
                 ("Q", (0, 3, 4), [(G(0, a, b), a, b) for b in K for a in K])]
    else:  # tet, StdTetExp.cpp:1075-1700
        verts = [G(0, 0, 0), G(1, 0, 0), G(0, 1, 0), G(0, 0, 1)]
        edges = [(0, 1, [(G(k, 0, 0), k) for k in K]), (1, 2, [(G(1, k - 1, 0), k) for k in K]),
                 (0, 2, [(G(0, k, 0), k) for k in K]), (0, 3, [(G(0, 0, k), k) for k in K]),
                 (1, 3, [(G(1, 0, k - 1), k) for k in K]), (2, 3, [(G(0, 1, k - 1), k) for k in K])]
        faces = [("T", (0, 1, 2), [(G(a, b, 0), a, b) for a in K for b in range(1, nm - a)]),
                 ("T", (0, 1, 3), [(G(a, 0, b), a, b) for a in K for b in range(1, nm - a)]),
                 ("T", (1, 2, 3), [(G(1, a - 1, b), a, b) for a in K for b in range(1, nm - a)]),
                 ("T", (0, 2, 3), [(G(0, a, b), a, b) for a in K for b in range(1, nm - a)])]
    return verts, edges, faces


def ncoeffs(shape, nm):
    return {"hex": nm ** 3, "prism": nm * nm * (nm + 1) // 2,
            "tet": nm * (nm + 1) * (nm + 2) // 6}[shape]


def _tables_1d(nm):
    """Modified_A at nm+1 GLL points and Modified_B at nm Gauss-Radau (1, 0)
    points with the raw weights (the face expansions' tables)."""
    import nektar_b200 as nb
    zg, wg, Dg = nb.points(nb.GLL, nm + 1)
    A, _ = nb.basis(nb.MODIFIED_A, nm, zg, Dg)
    zr, wr, Dr = nb.points(nb.RADAU_A1, nm)
    Bt, _ = nb.basis(nb.MODIFIED_B, nm, zr, Dr)
    Bt = np.asarray(Bt).reshape(-1, nm)
    rows, i = {}, 0
    for p in range(nm):
        for q in range(nm - p):
            rows[(p, q)] = Bt[i]
            i += 1
    return np.asarray(A).reshape(nm, nm + 1), zg, wg, rows, zr, wr * 0.5


# ---------------------------------------------------------------------------
# collections and the mesh
# ---------------------------------------------------------------------------

def _interp_matrix(zfrom, zto):
    """Lagrange interpolation from the points zfrom to the points zto
    (LibUtilities::Interp1D)."""
    n = len(zfrom)
    Vf = np.polynomial.legendre.legvander(zfrom, n - 1)
    Vt = np.polynomial.legendre.legvander(zto, n - 1)
    return Vt @ np.linalg.inv(Vf)


class Collection:
    """One operator collection: elements of one shape and order, with the
    attributes nektar_b200.Operator takes."""

    def __init__(self, geom, shape, nm, eids):
        self.shape, self.nm, self.elem_ids = shape, nm, list(eids)
        self.nelmt = len(self.elem_ids)
        self.T, self.nq = shape_tables(shape, nm, nm + 1)
        self.nt = self.nq[0] * self.nq[1] * self.nq[2]
        self.nc = ncoeffs(shape, nm)
        self.deformed = True
        self.lverts = np.array([local_vertices(geom, e) for e in self.elem_ids], dtype=np.int64)
        self.X = np.array([[geom.vertices[v] for v in row] for row in self.lverts])
        curves = None
        if geom.curved_edges:
            eid = {tuple(sorted(vs)): i for i, vs in geom.edges.items()}
            _, edges, _ = topology(shape, nm)
            curves = []
            for row in self.lverts:
                lst = []
                for a, b, _ in edges:
                    ge = eid.get(tuple(sorted((int(row[a]), int(row[b])))))
                    if ge in geom.curved_edges:
                        p = geom.curved_edges[ge]
                        lst.append(((a, b), 4.0 * (p[1] - 0.5 * (p[0] + p[2]))))
                curves.append(lst)
            self.deformed = True
        self.curves = curves
        fcurves = None
        if geom.curved_faces:
            fcurves = []
            for e in self.elem_ids:
                fcurves.append([(lf, face_bubble_coeff(geom.curved_faces[f]))
                                for lf, f in enumerate(geom.elements[e][1])
                                if f in geom.curved_faces and geom.faces[f][0] == "Q"])
        self.face_curves = fcurves
        self.jac, self.df, self.xyz = element_geometry(
            shape, self.X, tuple(np.asarray(z) for z in self.T["z"]), curves, fcurves)

    def quad_weights(self):
        """Integration weights jac * w0 w1 w2 at every quadrature point (the
        collapsed directions' Gauss-Radau weights carry the Duffy factor)."""
        w = [np.asarray(v) for v in self.T["ws"]]
        wq = np.einsum("k,j,i->kji", w[2], w[1], w[0]).reshape(-1)
        return self.jac * np.tile(wq, self.nelmt)


class SessionMesh:
    """The mesh of a session: collections (one per shape and order, in the
    order of the domain's composites), the assembly over the concatenated
    local coefficient vector and the Dirichlet data. With a single
    collection the object also carries that collection's attributes, so it
    can be handed to nektar_b200.Operator directly."""

    def __init__(self, session, var=None):
        g = session.geometry
        self.session = session
        self.var = var or (session.variables[0] if session.variables else "u")
        groups = {}
        for c in g.domain:
            letter, ids = g.composites[c]
            if letter not in ("H", "R", "A", "P"):
                raise SessionError("domain composite %d does not hold elements" % c)
            if c not in session.nummodes:
                raise SessionError("no expansion defined on composite %d" % c)
            for e in ids:
                shape = g.elements[e][0]
                groups.setdefault((shape, session.nummodes[c]), []).append(e)
        order = {"hex": 0, "prism": 1, "tet": 2}
        self.collections = [Collection(g, s, nm, ids) for (s, nm), ids in
                            sorted(groups.items(), key=lambda kv: (order[kv[0][0]], kv[0][1]))]
        self.offsets = np.cumsum([0] + [c.nelmt * c.nc for c in self.collections])
        self.nloc = int(self.offsets[-1])
        if len(self.collections) == 1:
            c = self.collections[0]
            for k in ("shape", "nm", "nq", "nt", "nc", "nelmt", "T", "deformed", "jac", "df",
                      "elem_ids", "lverts", "X"):
                setattr(self, k, getattr(c, k))
        self.xyz = np.concatenate([c.xyz for c in self.collections], axis=1)
        self._assemble()

    # ------------------------------------------------------------------ #
    def _dirichlet_faces(self):
        g, s = self.session.geometry, self.session
        self._face_bc = {}    # Dirichlet faces
        self._face_weak = {}  # Neumann and Robin faces (weak terms)
        for rid, comps in s.boundary_regions.items():
            conds = [bc for bc in s.boundary_conditions.get(rid, []) if bc.var == self.var]
            if not conds:
                continue
            bc = conds[0]
            if bc.kind not in ("D", "N", "R"):
                raise SessionError("boundary condition %r on region %d is not supported "
                                   % (bc.kind, rid))
            if bc.kind == "R" and bc.primcoeff is None:
                raise SessionError("Robin condition on region %d without PRIMCOEFF" % rid)
            for c in comps:
                letter, ids = g.composites[c]
                if letter not in ("F", "Q", "T"):
                    raise SessionError("boundary composite %d does not hold faces" % c)
                for f in ids:
                    (self._face_bc if bc.kind == "D" else self._face_weak)[f] = bc

    def _entity_orders(self):
        """Lowest order (modes) of the elements sharing each edge and face:
        with variable order an edge or face carries only the modes of its
        lowest-order element (AssemblyMapCG.cpp:1330-1375)."""
        low = {}
        for col in self.collections:
            _, edges, faces = topology(col.shape, col.nm)
            for el in range(col.nelmt):
                V = [int(v) for v in col.lverts[el]]
                keys = [("e", min(V[a], V[b]), max(V[a], V[b])) for a, b, _ in edges]
                for kind, frame, _ in faces:
                    if kind == "Q":
                        cs = {V[i] for i in frame} | {self._quad_of(col.shape, frame, V)}
                        keys.append(("f",) + tuple(sorted(cs)))
                    else:
                        keys.append(("t",) + tuple(sorted(V[i] for i in frame)))
                for k in keys:
                    low[k] = min(low.get(k, col.nm), col.nm)
        return low

    def _assemble(self):
        g = self.session.geometry
        self._dirichlet_faces()
        low = self._entity_orders()
        self.variable_order = len({c.nm for c in self.collections}) > 1
        entities = {}  # key -> size
        tri_frame = {}  # triangle key -> (apex, origin) of its canonical frame
        tri_pos = {}  # order -> {(a, b): position among a triangle's interior modes}
        gm, sg = [], []
        for col in self.collections:
            nm, nb = col.nm, col.nm - 2
            verts, edges, faces = topology(col.shape, nm)
            all_modes = set(verts)
            for _, _, lst in edges:
                all_modes.update(m for m, _ in lst)
            for _, _, lst in faces:
                all_modes.update(m for m, _, _ in lst)
            interior = [m for m in range(col.nc) if m not in all_modes]
            for el in range(col.nelmt):
                V = [int(v) for v in col.lverts[el]]
                key_of = [None] * col.nc
                for lv, m in enumerate(verts):
                    key_of[m] = (("v", V[lv]), 0, 1.0)
                    entities.setdefault(("v", V[lv]), 1)
                for a, b, lst in edges:
                    ga, gb = V[a], V[b]
                    key = ("e", min(ga, gb), max(ga, gb))
                    lo = low[key]
                    entities.setdefault(key, lo - 2)
                    for m, k in lst:
                        if k < lo:
                            key_of[m] = (key, k - 2, (-1.0) ** k if ga > gb else 1.0)
                        else:  # a mode the lower-order neighbour lacks: sign 0
                            key_of[m] = (("v", ga), 0, 0.0)
                for kind, frame, lst in faces:
                    if kind == "Q":
                        o, ea, eb = (V[i] for i in frame)
                        quad = self._quad_of(col.shape, frame, V)  # corner opposite o
                        cid = {(0, 0): o, (1, 0): ea, (0, 1): eb, (1, 1): quad}
                        key = ("f",) + tuple(sorted(cid.values()))
                        lb = low[key] - 2
                        entities.setdefault(key, lb * lb)
                        aO, bO = min(cid, key=lambda c: cid[c])
                        n1, n2 = cid[(1 - aO, bO)], cid[(aO, 1 - bO)]
                        s1 = 1 if aO == 0 else -1
                        s2 = 1 if bO == 0 else -1
                        for m, a, b in lst:
                            ca, cb = (a, b) if n1 < n2 else (b, a)
                            if ca - 2 < lb and cb - 2 < lb:
                                key_of[m] = (key, (ca - 2) * lb + (cb - 2),
                                             float(s1 ** a * s2 ** b))
                            else:
                                key_of[m] = (("v", o), 0, 0.0)
                    else:
                        o, ea, apex = (V[i] for i in frame)
                        key = ("t",) + tuple(sorted((o, ea, apex)))
                        lo = low[key]
                        entities.setdefault(key, (lo - 3) * (lo - 2) // 2)
                        if lo not in tri_pos:
                            tri_pos[lo] = {ab: i for i, ab in enumerate(
                                (a, b) for a in range(2, lo) for b in range(1, lo - a))}
                        tp = tri_pos[lo]
                        if key not in tri_frame:
                            tri_frame[key] = (apex, min(o, ea))
                        capex, corigin = tri_frame[key]
                        if capex != apex:
                            raise SessionError(
                                "triangular face %s: neighbouring elements collapse it towards "
                                "different vertices (%d, %d)" % (key[1:], capex, apex))
                        refl = o != corigin
                        for m, a, b in lst:
                            if (a, b) in tp:
                                key_of[m] = (key, tp[(a, b)], (-1.0) ** a if refl else 1.0)
                            else:
                                key_of[m] = (("v", o), 0, 0.0)
                for pos, m in enumerate(interior):
                    key_of[m] = (("i", len(gm), el), pos, 1.0)
                entities.setdefault(("i", len(gm), el), len(interior))
                gm.append(key_of)
        self._tri_frame = tri_frame
        # Dirichlet entities: the vertices, edges and faces of Dirichlet faces
        dir_ent = set()
        for f in self._face_bc:
            kind, es = g.faces[f]
            vs = sorted({v for e in es for v in g.edges[e]})
            dir_ent.add(("f" if kind == "Q" else "t",) + tuple(vs))
            for e in es:
                a, b = g.edges[e]
                dir_ent.update({("e", min(a, b), max(a, b)), ("v", a), ("v", b)})
        missing = [k for k in dir_ent if k not in entities]
        if missing:
            raise SessionError("boundary faces that belong to no element: %s" % missing[:3])
        rank = {"v": 0, "e": 1, "f": 2, "t": 3, "i": 4}
        keys = sorted(entities, key=lambda k: (k not in dir_ent, rank[k[0]], k[1:]))
        base, n, ndir = {}, 0, 0
        for k in keys:
            base[k] = n
            n += entities[k]
            if k in dir_ent:
                ndir = n
        self.nglob, self.ndir = n, ndir
        gmap = np.empty(self.nloc, dtype=np.int32)
        sign = np.empty(self.nloc)
        i = 0
        for key_of in gm:
            for key, off, s in key_of:
                gmap[i] = base[key] + off
                sign[i] = s
                i += 1
        self.gmap, self.sign = gmap, sign
        self._base, self._entities, self._dir_ent = base, entities, dir_ent

    @staticmethod
    def _quad_of(shape, frame, V):
        """The corner of a quadrilateral face opposite its frame origin."""
        opposite = {("hex", (0, 1, 3)): 2, ("hex", (0, 1, 4)): 5, ("hex", (1, 2, 5)): 6,
                    ("hex", (3, 2, 7)): 6, ("hex", (0, 3, 4)): 7, ("hex", (4, 5, 7)): 6,
                    ("prism", (0, 1, 3)): 2, ("prism", (1, 2, 4)): 5, ("prism", (0, 3, 4)): 5}
        return V[opposite[(shape, tuple(frame))]]

    # ------------------------------------------------------------------ #
    def dirichlet_values(self, time=0.0):
        """Global Dirichlet coefficients (ndir,) by the boundary-constrained
        projection of the boundary values."""
        g = self.session.geometry
        nms = {c.nm for c in self.collections}
        if len(nms) != 1:
            raise SessionError("consistent Dirichlet values with several expansion orders are "
                               "not supported (dirichlet_local takes them)")
        nm = nms.pop()
        nb = nm - 2
        A, zg, wg, Brow, zr, wr = _tables_1d(nm)
        out = np.zeros(self.ndir)
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        ent_bc = {}
        for f, bc in self._face_bc.items():
            for e in g.faces[f][1]:
                a, b = g.edges[e]
                ent_bc.setdefault(("v", a), bc)
                ent_bc.setdefault(("v", b), bc)
                ent_bc.setdefault(("e", min(a, b), max(a, b)), bc)
        vals = {}
        for key, bc in ent_bc.items():
            if key[0] == "v":
                x = P(key[1])
                vals[key[1]] = out[self._base[key]] = bc.value.evaluate(x[0], x[1], x[2], time)
        M1 = (A[2:] * wg) @ A[2:].T
        for key, bc in ent_bc.items():
            if key[0] != "e" or nb == 0:
                continue
            xa, xb = P(key[1]), P(key[2])
            x = np.outer(0.5 * (1 - zg), xa) + np.outer(0.5 * (1 + zg), xb)
            f = bc.value.evaluate(x[:, 0], x[:, 1], x[:, 2], time)
            rem = f - f[0] * A[0] - f[-1] * A[1]
            o = self._base[key]
            out[o:o + nb] = np.linalg.solve(M1, (A[2:] * wg) @ rem)

        def edge_coeffs(a, b):
            k = ("e", min(a, b), max(a, b))
            c = out[self._base[k]:self._base[k] + nb].copy()
            if a > b:  # face direction runs against the edge's numbering
                c *= (-1.0) ** np.arange(2, nm)
            return c

        for f, bc in self._face_bc.items():
            kind, es = g.faces[f]
            if nb == 0:
                continue
            if kind == "Q":
                self._quad_face(f, bc, time, out, vals, edge_coeffs, A, zg, wg, nm)
            else:
                self._tri_face(f, bc, time, out, vals, edge_coeffs, A, zg, wg, Brow, zr, wr, nm)
        return out

    def _quad_face(self, f, bc, time, out, vals, edge_coeffs, A, z, w, nm):
        g = self.session.geometry
        nb = nm - 2
        cyc = self._face_cycle(f)
        i0 = int(np.argmin(cyc))
        O = cyc[i0]
        nA, nB = cyc[(i0 + 1) % 4], cyc[(i0 - 1) % 4]
        if nA > nB:
            nA, nB = nB, nA
        AB = cyc[(i0 + 2) % 4]
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        za, zb = np.meshgrid(z, z, indexing="ij")
        x, J = self._quad_map(O, nA, nB, AB, za, zb)
        fv = bc.value.evaluate(x[..., 0], x[..., 1], x[..., 2], time)
        ub = (vals[O] * np.outer(A[0], A[0]) + vals[nA] * np.outer(A[1], A[0])
              + vals[nB] * np.outer(A[0], A[1]) + vals[AB] * np.outer(A[1], A[1]))
        for (a, b, side, along) in ((O, nA, 0, "a"), (nB, AB, 1, "a"), (O, nB, 0, "b"),
                                    (nA, AB, 1, "b")):
            prof = edge_coeffs(a, b) @ A[2:]
            ub = ub + (np.outer(prof, A[side]) if along == "a" else np.outer(A[side], prof))
        W = np.outer(w, w) * J
        Bi = A[2:]
        rhs = np.einsum("ai,bj,ij->ab", Bi, Bi, W * (fv - ub)).reshape(-1)
        M2 = np.einsum("ai,ci,bj,dj,ij->abcd", Bi, Bi, Bi, Bi, W).reshape(nb * nb, nb * nb)
        key = ("f",) + tuple(sorted(cyc))
        o = self._base[key]
        out[o:o + nb * nb] = np.linalg.solve(M2, rhs)

    def _tri_face(self, f, bc, time, out, vals, edge_coeffs, A, zs, ws, Brow, zt, wt, nm):
        """Constrained projection on a triangle in its canonical frame
        (origin, end of axis a, apex): modes phi_p(s) psi_pq(t), the apex
        vertex mode psi_01(t) (the collapsed-vertex fix of StdTriExp)."""
        g = self.session.geometry
        vs = sorted({v for e in g.faces[f][1] for v in g.edges[e]})
        key = ("t",) + tuple(vs)
        apex, O = self._tri_frame[key]
        E = [v for v in vs if v not in (apex, O)][0]
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        XO, XE, XC = P(O), P(E), P(apex)
        S, T = np.meshgrid(zs, zt, indexing="ij")  # [i (s), j (t)]
        xa = 0.5 * (1 + S) * (1 - T) - 1
        xb = T
        x = (-0.5 * (xa + xb))[..., None] * XO + (0.5 * (1 + xa))[..., None] * XE + \
            (0.5 * (1 + xb))[..., None] * XC
        J = np.linalg.norm(np.cross(0.5 * (XE - XO), 0.5 * (XC - XO)))
        fv = bc.value.evaluate(x[..., 0], x[..., 1], x[..., 2], time)
        phi = A  # (nm, nq_s)
        ub = (vals[O] * np.outer(phi[0], Brow[(0, 0)]) + vals[E] * np.outer(phi[1], Brow[(1, 0)])
              + vals[apex] * np.outer(np.ones_like(zs), Brow[(0, 1)]))
        for k, c in zip(range(2, nm), edge_coeffs(O, E)):
            ub = ub + c * np.outer(phi[k], Brow[(k, 0)])
        for k, c in zip(range(2, nm), edge_coeffs(O, apex)):
            ub = ub + c * np.outer(phi[0], Brow[(0, k)])
        for k, c in zip(range(2, nm), edge_coeffs(E, apex)):
            ub = ub + c * np.outer(phi[1], Brow[(1, k - 1)])
        modes = [(a, b) for a in range(2, nm) for b in range(1, nm - a)]
        if not modes:
            return
        F = np.stack([np.outer(phi[a], Brow[(a, b)]) for a, b in modes])  # (nmodes, s, t)
        W = np.outer(ws, wt) * J
        rhs = np.einsum("mij,ij->m", F, W * (fv - ub))
        M = np.einsum("mij,nij,ij->mn", F, F, W)
        o = self._base[key]
        out[o:o + len(modes)] = np.linalg.solve(M, rhs)

    def _curve(self, a, b):
        """Mode-2 coefficient (3,) of the edge between global vertices a and
        b: 4 (midpoint - mean of the ends) for a quadratic curved edge
        (SegGeom::v_FillGeom projects the curve on the edge's modes), zero
        for a straight one. The same for either direction."""
        g = self.session.geometry
        if not g.curved_edges:
            return np.zeros(3)
        if not hasattr(self, "_edge_of"):
            self._edge_of = {tuple(sorted(vs)): i for i, vs in g.edges.items()}
        e = self._edge_of.get(tuple(sorted((a, b))))
        if e not in g.curved_edges:
            return np.zeros(3)
        p = g.curved_edges[e]
        return 4.0 * (p[1] - 0.5 * (p[0] + p[2]))

    def _edge_points(self, a, b, s):
        P = lambda v: np.asarray(self.session.geometry.vertices[v], dtype=np.float64)  # noqa: E731
        return np.outer(0.5 * (1 - s), P(a)) + np.outer(0.5 * (1 + s), P(b)) + \
            np.outer(0.25 * (1 - s * s), self._curve(a, b))

    def _edge_speed(self, a, b, s):
        P = lambda v: np.asarray(self.session.geometry.vertices[v], dtype=np.float64)  # noqa: E731
        d = 0.5 * (P(b) - P(a))[None, :] - np.outer(0.5 * s, self._curve(a, b))
        return np.linalg.norm(d, axis=1)

    def _face_curve(self, vs):
        """(2, 2) coefficient (3,) of the quadrilateral face with global
        vertices vs if it is curved, else zero."""
        g = self.session.geometry
        if not g.curved_faces:
            return np.zeros(3)
        if not hasattr(self, "_face_of"):
            self._face_of = {frozenset(v for e in es for v in g.edges[e]): f
                             for f, (kind, es) in g.faces.items() if kind == "Q"}
        f = self._face_of.get(frozenset(vs))
        if f not in g.curved_faces:
            return np.zeros(3)
        return face_bubble_coeff(g.curved_faces[f])

    def _quad_map(self, O, nA, nB, AB, za, zb):
        """Points and surface Jacobian of the quadrilateral face O, nA, AB, nB
        (coordinates za along O -> nA, zb along O -> nB): the bilinear map
        plus the quadratic curves of its edges and of the face itself."""
        P = lambda v: np.asarray(self.session.geometry.vertices[v], dtype=np.float64)  # noqa: E731
        XO, XA, XB, XAB = P(O), P(nA), P(nB), P(AB)
        Na = [0.5 * (1 - za), 0.5 * (1 + za)]
        Nb = [0.5 * (1 - zb), 0.5 * (1 + zb)]
        x = (Na[0] * Nb[0])[..., None] * XO + (Na[1] * Nb[0])[..., None] * XA + \
            (Na[0] * Nb[1])[..., None] * XB + (Na[1] * Nb[1])[..., None] * XAB
        dxa = (0.5 * Nb[0])[..., None] * (XA - XO) + (0.5 * Nb[1])[..., None] * (XAB - XB)
        dxb = (0.5 * Na[0])[..., None] * (XB - XO) + (0.5 * Na[1])[..., None] * (XAB - XA)
        for p, q, t, u, along in ((O, nA, za, Nb[0], "a"), (nB, AB, za, Nb[1], "a"),
                                  (O, nB, zb, Na[0], "b"), (nA, AB, zb, Na[1], "b")):
            c = self._curve(p, q)
            if not c.any():
                continue
            bub, dbub = 0.25 * (1 - t * t), -0.5 * t
            du = -0.5 if u is Nb[0] or u is Na[0] else 0.5
            x = x + (bub * u)[..., None] * c
            if along == "a":
                dxa = dxa + (dbub * u)[..., None] * c
                dxb = dxb + (bub * du)[..., None] * c
            else:
                dxb = dxb + (dbub * u)[..., None] * c
                dxa = dxa + (bub * du)[..., None] * c
        cf = self._face_curve((O, nA, nB, AB))
        if cf.any():
            ba, bb = 0.25 * (1 - za * za), 0.25 * (1 - zb * zb)
            x = x + (ba * bb)[..., None] * cf
            dxa = dxa + (-0.5 * za * bb)[..., None] * cf
            dxb = dxb + (ba * -0.5 * zb)[..., None] * cf
        return x, np.linalg.norm(np.cross(dxa, dxb), axis=-1)

    def _tri_map(self, v0, v1, v2, xa, xb):
        """Points and surface Jacobian (per unit d xa d xb) of the triangle
        v0, v1, v2 at its standard coordinates: the linear map plus the
        quadratic curves of its edges (products of the end barycentrics)."""
        P = lambda v: np.asarray(self.session.geometry.vertices[v], dtype=np.float64)  # noqa: E731
        lam = [-0.5 * (xa + xb), 0.5 * (1 + xa), 0.5 * (1 + xb)]
        dl = [(-0.5, -0.5), (0.5, 0.0), (0.0, 0.5)]
        V = [v0, v1, v2]
        x = sum(lam[i][..., None] * P(V[i]) for i in range(3))
        dxa = sum(dl[i][0] * P(V[i]) for i in range(3)) + 0 * x
        dxb = sum(dl[i][1] * P(V[i]) for i in range(3)) + 0 * x
        for i, j in ((0, 1), (1, 2), (0, 2)):
            c = self._curve(V[i], V[j])
            if not c.any():
                continue
            x = x + (lam[i] * lam[j])[..., None] * c
            dxa = dxa + (dl[i][0] * lam[j] + dl[j][0] * lam[i])[..., None] * c
            dxb = dxb + (dl[i][1] * lam[j] + dl[j][1] * lam[i])[..., None] * c
        return x, np.linalg.norm(np.cross(dxa, dxb), axis=-1)

    def _face_cycle(self, f):
        """The global vertex ids of face f in cyclic order."""
        g = self.session.geometry
        es = [g.edges[e] for e in g.faces[f][1]]
        cyc = [es[0][0], es[0][1]]
        n = len(es)
        while len(cyc) < n:
            last = cyc[-1]
            for a, b in es:
                if a == last and b not in cyc:
                    cyc.append(b)
                    break
                if b == last and a not in cyc:
                    cyc.append(a)
                    break
            else:
                raise SessionError("face %d is not a closed cycle" % f)
        return cyc

    def dirichlet_local(self, time=0.0, consistent=False):
        """Local coefficient vector holding the Dirichlet values (zeros
        elsewhere), the x_loc a solve takes for the lifting.

        By default built as ContField::v_ImposeDirichletConditions builds it
        in a serial run (ContField.cpp:557-613): every Dirichlet boundary
        face, in boundary-region, composite and listed order, projects the
        data with its own expansion's FwdTransBndConstrained in its own frame
        and writes the result into its element's local coefficients, later
        faces overwriting shared vertex and edge modes (the max-abs merge of
        :602 only acts across partitions). On a triangle
        (TriExp::v_FwdTransBndConstrained) the data of edges 1 and 2 are
        interpolated from the Gauss-Radau points to GLL points before their
        1-D projection and edge 2 is written last, so the apex value is the
        extrapolation along edge 2. consistent=True instead takes one global
        value per Dirichlet dof (dirichlet_values)."""
        x = np.zeros(self.nloc)
        mask = self.gmap < self.ndir
        if consistent:
            dv = self.dirichlet_values(time)
            x[mask] = self.sign[mask] * dv[self.gmap[mask]]
            return x
        owner = self._face_owners()
        g, s = self.session.geometry, self.session
        written, src = np.zeros(self.nloc, dtype=bool), {}
        for f in self._boundary_face_order():
            if f not in self._face_bc:
                continue
            lo, hi, nm = owner[f]
            vals = self._face_values(f, self._face_bc[f], time, nm)
            gm, sg = self.gmap[lo:hi], self.sign[lo:hi]
            for i, gd in enumerate(gm):
                # modes a lower-order neighbour lacks (sign 0) end up zero and
                # are no source for other copies (AssemblyMapCG.cpp:1940-1957)
                if gd in vals and sg[i] != 0.0:
                    x[lo + i] = sg[i] * vals[gd]
                    written[lo + i] = True
                    src[int(gd)] = lo + i  # the last write of each dof
        # local copies of Dirichlet dofs on elements that touch the boundary
        # only at an edge or vertex take the last written copy's value
        # (AssemblyMapCG.cpp:1925-2010, the copyLocalDirDofs of :609-613)
        for k in np.nonzero(mask & ~written)[0]:
            j = src[int(self.gmap[k])]
            x[k] = x[j] * self.sign[j] * self.sign[k]
        return x

    def _boundary_face_order(self):
        """Dirichlet faces in the order of the reference's boundary expansions:
        regions in id order; within a region its composites in id order, the
        faces grouped by expansion type (basis and regular / deformed
        geometry) in order of first appearance, listed order within a group
        (ExpList's CompositeMap constructor, ExpList.cpp:1436-1462)."""
        g, s = self.session.geometry, self.session
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        out = []
        for rid in sorted(s.boundary_regions):
            groups = {}
            for c in sorted(s.boundary_regions[rid]):
                if c not in g.composites:
                    continue
                for f in g.composites[c][1]:
                    kind = g.faces[f][0]
                    regular = not any(e in g.curved_edges for e in g.faces[f][1]) and \
                        f not in g.curved_faces
                    if kind == "Q" and regular:  # a parallelogram has a constant Jacobian
                        cyc = [P(v) for v in self._face_cycle(f)]
                        regular = bool(np.allclose(cyc[0] + cyc[2], cyc[1] + cyc[3],
                                                   rtol=0, atol=1e-12))
                    groups.setdefault((kind, regular), []).append(f)
            for lst in groups.values():  # dicts keep first-appearance order
                out.extend(lst)
        return out

    def _face_owners(self):
        """Local coefficient range and order of the element that owns each
        boundary face."""
        g = self.session.geometry
        out = {}
        for ci, col in enumerate(self.collections):
            base = int(self.offsets[ci])
            for el, eid in enumerate(col.elem_ids):
                for f in g.elements[eid][1]:
                    if f in self._face_bc or f in self._face_weak:
                        out[f] = (base + el * col.nc, base + (el + 1) * col.nc, col.nm)
        return out

    # ------------------------------------------------------------------ #
    def _quad_face_basis(self, f, nm):
        """Quadrature of the quadrilateral boundary face f at its element's
        order (nm modes, nm+1 GLL points per direction, the trace expansion's)
        and the global basis functions living on it: (x [3, q, q], weights
        with the surface Jacobian [q, q], global dofs, values [ndof, q, q]).
        The functions are the global ones of the assembly: vertex modes,
        edge modes along the edge's lower -> higher vertex id (its modes a
        lower-order neighbour lacks left out), face modes in the face's
        canonical frame (origin the lowest vertex, first axis towards its
        lower-id neighbour)."""
        g = self.session.geometry
        A, zg, wg, _, _, _ = _tables_1d(nm)
        cyc = self._face_cycle(f)
        i0 = int(np.argmin(cyc))
        O = cyc[i0]
        nA, nB = sorted((cyc[(i0 + 1) % 4], cyc[(i0 - 1) % 4]))
        AB = cyc[(i0 + 2) % 4]
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        za, zb = np.meshgrid(zg, zg, indexing="ij")
        x, J = self._quad_map(O, nA, nB, AB, za, zb)
        W = np.outer(wg, wg) * J
        dofs, F = [], []
        for v, (i, j) in ((O, (0, 0)), (nA, (1, 0)), (nB, (0, 1)), (AB, (1, 1))):
            dofs.append(self._base[("v", v)])
            F.append(np.outer(A[i], A[j]))
        for p, q, side, along in ((O, nA, 0, "a"), (O, nB, 0, "b"), (nA, AB, 1, "b"),
                                  (nB, AB, 1, "a")):
            key = ("e", min(p, q), max(p, q))
            o, size = self._base[key], self._entities[key]
            for k in range(2, min(nm, size + 2)):
                sg = 1.0 if p < q else (-1.0) ** k
                dofs.append(o + k - 2)
                F.append(sg * (np.outer(A[k], A[side]) if along == "a"
                               else np.outer(A[side], A[k])))
        key = ("f",) + tuple(sorted(cyc))
        o, lb = self._base[key], int(round(self._entities[key] ** 0.5))
        for a in range(2, min(nm, lb + 2)):
            for b in range(2, min(nm, lb + 2)):
                dofs.append(o + (a - 2) * lb + (b - 2))
                F.append(np.outer(A[a], A[b]))
        return x.transpose(2, 0, 1), W, np.array(dofs, dtype=np.int64), np.array(F)

    def _tri_face_basis(self, f, nm):
        """_quad_face_basis for a triangular face: its canonical frame
        (origin, end of the first axis, the apex its elements collapse
        towards), the trace expansion's points (GLL nm+1 along the first
        axis, Gauss-Radau (1, 0) nm towards the apex), and the global
        functions on it: vertex modes (the apex mode the collapsed psi_01),
        edge modes along each edge's lower -> higher vertex id, face modes
        phi_a psi_ab in the canonical frame."""
        g = self.session.geometry
        A, zg, wg, Brow, zr, wr = _tables_1d(nm)
        vs = sorted({v for e in g.faces[f][1] for v in g.edges[e]})
        key = ("t",) + tuple(vs)
        C, O = self._tri_frame[key]
        E = [v for v in vs if v not in (C, O)][0]
        S, T = np.meshgrid(zg, zr, indexing="ij")
        xa = 0.5 * (1 + S) * (1 - T) - 1
        x, Jt = self._tri_map(O, E, C, xa, T)
        W = np.outer(wg, wr) * Jt
        ones = np.ones_like(zg)
        dofs = [self._base[("v", O)], self._base[("v", E)], self._base[("v", C)]]
        F = [np.outer(A[0], Brow[(0, 0)]), np.outer(A[1], Brow[(1, 0)]),
             np.outer(ones, Brow[(0, 1)])]
        for p, q, fn in ((O, E, lambda k: np.outer(A[k], Brow[(k, 0)])),
                         (O, C, lambda k: np.outer(A[0], Brow[(0, k)])),
                         (E, C, lambda k: np.outer(A[1], Brow[(1, k - 1)]))):
            ek = ("e", min(p, q), max(p, q))
            o, size = self._base[ek], self._entities[ek]
            for k in range(2, min(nm, size + 2)):
                dofs.append(o + k - 2)
                F.append((1.0 if p < q else (-1.0) ** k) * fn(k))
        o = self._base[key]
        lo = int(round(0.5 * (5 + (1 + 8 * self._entities[key]) ** 0.5)))  # the face's order
        pos = 0
        for a in range(2, lo):
            for b in range(1, lo - a):
                dofs.append(o + pos)
                F.append(np.outer(A[a], Brow[(a, b)]))
                pos += 1
        return x.transpose(2, 0, 1), W, np.array(dofs, dtype=np.int64), np.array(F)

    def weak_terms(self, time=0.0):
        """The Neumann and Robin terms of the Helmholtz system
        (ContField::v_HelmSolve, ContField.cpp:822-855: the boundary
        expansions' inner products of the data added to the forcing;
        Expansion3D::v_AddRobinMassMatrix / AddRobinTraceContribution,
        Expansion3D.cpp:2045-: PRIMCOEFF-weighted face mass matrices added to
        the operator, GlobalLinSysIterativeFull.cpp:133-150,213-231).
        Returns (local right-hand side contribution [nloc], Robin blocks
        [(global dofs, matrix, owner local indices)])."""
        g = self.session.geometry
        rhs = np.zeros(self.nloc)
        robin = []
        if not self._face_weak:
            return rhs, robin
        owner = self._face_owners()
        for f, bc in self._face_weak.items():
            lo, hi, nm = owner[f]
            if g.faces[f][0] == "Q":
                x, W, dofs, F = self._quad_face_basis(f, nm)
            else:
                x, W, dofs, F = self._tri_face_basis(f, nm)
            gl = self.gmap[lo:hi]
            loc = np.empty(dofs.size, dtype=np.int64)
            for i, d in enumerate(dofs):
                hit = np.nonzero((gl == d) & (self.sign[lo:hi] != 0))[0]
                loc[i] = lo + hit[0]
            gv = bc.value.evaluate(x[0], x[1], x[2], time)
            np.add.at(rhs, loc, self.sign[loc] * np.einsum("mij,ij->m", F, W * gv))
            if bc.kind == "R":
                al = np.broadcast_to(bc.primcoeff.evaluate(x[0], x[1], x[2], time), W.shape)
                robin.append((dofs, np.einsum("mij,nij,ij->mn", F, F, W * al), loc))
        return rhs, robin

    def _face_values(self, f, bc, time, nm):
        """{global dof: value} of the Dirichlet face f's boundary-constrained
        projection, as the face's own expansion (nm modes, its element's)
        computes it; an edge shared with lower-order elements keeps its
        lower modes only."""
        g = self.session.geometry
        nb = nm - 2
        A, zg, wg, Brow, zr, wr = _tables_1d(nm)
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        kind, es = g.faces[f]
        E = [g.edges[e] for e in es]
        # the face's own frame: vertex j starts edge j (TriGeom / QuadGeom)
        fv = []
        for j in range(len(E)):
            a, b = E[j]
            nxt = E[(j + 1) % len(E)]
            fv.append(a if b in nxt else b)
        vals = {}

        def proj1d(data, a=None, b=None):
            """SegExp::FwdTransBndConstrained of edge data at the GLL points:
            vertex values, then the L2 projection of the rest onto the
            interior modes with the edge's Jacobian (|dx/ds|, not constant on
            a curved edge)."""
            c = np.zeros(nm)
            c[0], c[1] = data[0], data[-1]
            if nb:
                js = np.ones_like(zg) if a is None else self._edge_speed(a, b, zg)
                wj = wg * js
                rem = data - c[0] * A[0] - c[1] * A[1]
                c[2:] = np.linalg.solve((A[2:] * wj) @ A[2:].T, (A[2:] * wj) @ rem)
            return c

        full = {}  # (a, b) -> the edge's coefficients along a -> b, all nm modes

        def put_edge(a, b, c):
            key = ("e", min(a, b), max(a, b))
            o = self._base[key]
            full[(a, b)] = c[2:]
            full[(b, a)] = c[2:] * (-1.0) ** np.arange(2, nm)
            cc = c[2:] * ((-1.0) ** np.arange(2, nm) if a > b else 1.0)
            for k in range(min(nb, self._entities[key])):
                vals[o + k] = cc[k]

        bcv = lambda x: bc.value.evaluate(x[..., 0], x[..., 1], x[..., 2], time)  # noqa: E731
        if kind == "Q":
            # symmetric GLL points: the same polynomial in every frame
            for v in fv:
                vals[self._base[("v", v)]] = float(bcv(P(v)))
            for j in range(4):
                a, b = fv[j], fv[(j + 1) % 4]
                x = self._edge_points(a, b, zg)
                put_edge(a, b, proj1d(bcv(x), a, b))
            if nb:
                out = np.zeros(self.ndir)
                for gd, v in vals.items():
                    out[gd] = v
                vtab = {v: vals[self._base[("v", v)]] for v in fv}

                def ec(a, b):
                    return full[(a, b)]
                self._quad_face(f, bc, time, out, vtab, ec, A, zg, wg, nm)
                key = ("f",) + tuple(sorted(fv))
                o = self._base[key]
                for k in range(nb * nb):
                    vals[o + k] = out[o + k]
            return vals
        # triangle in its own frame: v0 -> v1 along s, apex v2 along t
        v0, v1, v2 = fv
        X0, X1, X2 = P(v0), P(v1), P(v2)
        S, T = np.meshgrid(zg, zr, indexing="ij")
        xa = 0.5 * (1 + S) * (1 - T) - 1
        x, Jt = self._tri_map(v0, v1, v2, xa, T)
        data = bcv(x)  # [s, t]
        I = _interp_matrix(zr, zg)  # Gauss-Radau -> GLL
        c0 = proj1d(data[:, 0], v0, v1)
        c1 = proj1d(I @ data[-1, :], v1, v2)
        c2 = proj1d(I @ data[0, :], v0, v2)
        vtab = {v0: c2[0], v1: c1[0], v2: c2[1]}  # edge 2 written last
        vtab[v1] = c1[0]
        for v, val in vtab.items():
            vals[self._base[("v", v)]] = val
        put_edge(v0, v1, c0)
        put_edge(v1, v2, c1)
        put_edge(v0, v2, c2)
        key = ("t",) + tuple(sorted(fv))
        capex, corigin = self._tri_frame[key]
        if capex != v2:
            raise SessionError("boundary triangle %d collapses towards %d, its element towards %d"
                               % (f, v2, capex))
        modes = [(a, b) for a in range(2, nm) for b in range(1, nm - a)]
        if modes:
            phi = A
            ub = (vtab[v0] * np.outer(phi[0], Brow[(0, 0)]) + vtab[v1] * np.outer(phi[1], Brow[(1, 0)])
                  + vtab[v2] * np.outer(np.ones_like(zg), Brow[(0, 1)]))
            for k in range(2, nm):
                ub = ub + c0[k] * np.outer(phi[k], Brow[(k, 0)]) \
                    + c2[k] * np.outer(phi[0], Brow[(0, k)]) + c1[k] * np.outer(phi[1], Brow[(1, k - 1)])
            F = np.stack([np.outer(phi[a], Brow[(a, b)]) for a, b in modes])
            W = np.outer(wg, wr) * Jt
            c = np.linalg.solve(np.einsum("mij,nij,ij->mn", F, F, W),
                                np.einsum("mij,ij->m", F, W * (data - ub)))
            refl = v0 != corigin
            o = self._base[key]
            for pos, (a, b) in enumerate(modes):
                vals[o + pos] = c[pos] * ((-1.0) ** a if refl else 1.0)
        return vals

    def quad_weights(self):
        return np.concatenate([c.quad_weights() for c in self.collections])

    def split(self, vec, per="coeff"):
        """Per-collection views of a concatenated local (coeff) or physical
        (phys) vector."""
        if per == "coeff":
            return [vec[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.collections))]
        off = np.cumsum([0] + [c.nelmt * c.nt for c in self.collections])
        return [vec[off[i]:off[i + 1]] for i in range(len(self.collections))]
