"""Mesh graph of a session for the B200 path: element frames, geometric
factors at the quadrature points, the C0 local -> global map with
Dirichlet degrees of freedom first, and the Dirichlet values.

Hexahedra, as the reference sets them up:

* local frame: HexGeom::SetUpLocalEdges / SetUpLocalVertices
  (SpatialDomains/HexGeom.cpp:200-430). The element lists its faces bottom,
  four sides, top; local edges are the faces' shared edges in a fixed
  order; local vertices follow the edge chain. Vertex v0 is xi = (-1,-1,-1),
  v1 (+1,-1,-1), v2 (+1,+1,-1), v3 (-1,+1,-1), v4..v7 the same at xi3 = +1;
* geometry: the straight-sided map is trilinear in the vertices (the
  two-mode coordinate expansion of Geometry3D); jac and df as GeomFactors
  defines them (GeomFactors.cpp:248-477), df[k*3+j] = d xi_j / d x_k, in the
  Collections layout (9, nelmt*nt);
* coefficients: Modified_A in each direction, mode (p, q, r) at
  p + nm (q + nm r); index 0 / 1 are the vertex modes at xi = -1 / +1,
  indices >= 2 the bubbles.

Continuity (the role of AssemblyMapCG, AssemblyMapCG.cpp:1322-2300): a local
mode is a vertex, edge, face or interior mode by how many of its indices are
bubbles. Edge modes are numbered along the edge from its lower to its higher
global vertex id; mode p of an element edge running the other way gets the
sign (-1)^p (the bubble phi_p(-xi) = (-1)^p phi_p(xi)). Face modes are
numbered in a frame anchored at the face's lowest global vertex, first axis
towards the lower of its two neighbours; an element face frame maps to it by
a transposition and two reflections, which permute the (a, b) mode indices
and give the sign (-1)^(a s_a + b s_b). Any consistent choice gives the same
discrete space as the reference's, hence the same solution.

Dirichlet values follow ExpList::FwdTransBndConstrained on the boundary
faces (QuadExp.cpp:67-170, SegExp.cpp:81-180): vertex modes take the point
values, edge bubbles the L2 projection (edge quadrature) of the remainder
after the vertex modes, face bubbles the L2 projection (face quadrature and
surface Jacobian) of the remainder after vertex and edge modes. The result
is independent of the face's parametrisation for the symmetric GLL points.
"""
import numpy as np

from . import shape_tables
from .session import SessionError

# local vertex index of the corner (a, b, c) in {0, 1}^3 (xi = 2a - 1, ...)
HEX_CORNER = {(0, 0, 0): 0, (1, 0, 0): 1, (1, 1, 0): 2, (0, 1, 0): 3,
              (0, 0, 1): 4, (1, 0, 1): 5, (1, 1, 1): 6, (0, 1, 1): 7}
HEX_CORNER_XI = np.array([[2 * a - 1, 2 * b - 1, 2 * c - 1]
                          for (a, b, c), _ in sorted(HEX_CORNER.items(), key=lambda kv: kv[1])],
                         dtype=np.float64)


def _shared_edge(fa, fb, faces, what):
    common = [e for e in faces[fa][1] if e in faces[fb][1]]
    if len(common) != 1:
        raise SessionError("faces %d and %d share %d edges (%s)" % (fa, fb, len(common), what))
    return common[0]


def hex_local_vertices(geom, eid):
    """Global vertex ids v0..v7 of hexahedron eid in its local order
    (HexGeom::SetUpLocalEdges, HexGeom.cpp:200-339, and
    HexGeom::SetUpLocalVertices, HexGeom.cpp:341-430)."""
    shape, F = geom.elements[eid]
    if shape != "hex" or len(F) != 6:
        raise SessionError("element %d is not a hexahedron" % eid)
    for f in F:
        if geom.faces[f][0] != "Q":
            raise SessionError("hexahedron %d has a non-quadrilateral face" % eid)
    faces = geom.faces
    e = [None] * 12
    for f in range(1, 5):
        e[f - 1] = _shared_edge(F[0], F[f], faces, "bottom")
    e[4] = _shared_edge(F[1], F[4], faces, "vertical")
    for f in range(1, 4):
        e[f + 4] = _shared_edge(F[f], F[f + 1], faces, "vertical")
    for f in range(1, 5):
        e[f + 7] = _shared_edge(F[5], F[f], faces, "top")
    E = [geom.edges[k] for k in e]

    def chain(first, second, nxt):
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

    return chain(0, 1, (1, 2)) + chain(8, 9, (9, 10))


def hex_geometry(X, z):
    """jac (nelmt*nt,), df (9, nelmt*nt) and coordinates (3, nelmt*nt) of
    trilinear hexahedra with corner coordinates X (nelmt, 8, 3) at the tensor
    points z (each direction the same, point q = (k nq + j) nq + i)."""
    nq = len(z)
    xi = np.stack(np.meshgrid(z, z, z, indexing="ij"), axis=-1)  # [i, j, k, dir]
    xi = xi.transpose(2, 1, 0, 3).reshape(-1, 3)  # q = (k nq + j) nq + i
    s = HEX_CORNER_XI  # (8, 3)
    fac = 0.5 * (1.0 + xi[:, None, :] * s[None, :, :])  # (nt, 8, 3)
    N = fac.prod(axis=2)  # (nt, 8)
    dN = np.empty((xi.shape[0], 8, 3))
    for j in range(3):
        d = fac.copy()
        d[:, :, j] = 0.5 * s[None, :, j]
        dN[:, :, j] = d.prod(axis=2)
    x = np.einsum("pc,ecd->edp", N, X)  # (nelmt, 3, nt)
    J = np.einsum("pcj,ecd->epdj", dN, X)  # J[e, p, d, j] = d x_d / d xi_j
    det = np.linalg.det(J)
    if np.any(det <= 0):
        raise SessionError("element with a non-positive Jacobian")
    inv = np.linalg.inv(J)  # inv[e, p, j, k] = d xi_j / d x_k
    ne, nt = X.shape[0], xi.shape[0]
    df = np.empty((9, ne * nt))
    for k in range(3):
        for j in range(3):
            df[k * 3 + j] = inv[:, :, j, k].reshape(-1)
    coords = x.transpose(1, 0, 2).reshape(3, -1)
    return det.reshape(-1), df, coords


def _modA(T):
    """(nm, nq) Modified_A table of direction 0 and its raw weights / points."""
    nq = len(T["z"][0])
    return np.asarray(T["b"][0]).reshape(-1, nq), np.asarray(T["w"][0]), np.asarray(T["z"][0])


class SessionMesh:
    """The hexahedral mesh of a session with the attributes the operators take
    (shape, nm, nq, nt, nc, nelmt, T, jac, df, deformed) plus coordinates of
    the quadrature points, the assembly and the Dirichlet data."""

    def __init__(self, session, var=None):
        g = session.geometry
        self.session = session
        self.var = var or (session.variables[0] if session.variables else "u")
        eids, nms = [], set()
        for c in g.domain:
            letter, ids = g.composites[c]
            if letter not in ("H", "R", "A", "P"):
                raise SessionError("domain composite %d does not hold elements" % c)
            if c not in session.nummodes:
                raise SessionError("no expansion defined on composite %d" % c)
            nms.add(session.nummodes[c])
            eids.extend(ids)
        shapes = {g.elements[e][0] for e in eids}
        if shapes != {"hex"}:
            raise SessionError("only hexahedral meshes are supported, found %s" % sorted(shapes))
        if len(nms) != 1:
            raise SessionError("one expansion order per mesh is supported")
        self.shape, self.nm = "hex", nms.pop()
        self.elem_ids = eids
        self.nelmt = len(eids)
        self.T, self.nq = shape_tables("hex", self.nm, self.nm + 1)
        self.nt = self.nq[0] * self.nq[1] * self.nq[2]
        self.nc = self.nm ** 3
        self.deformed = True
        self.lverts = np.array([hex_local_vertices(g, e) for e in eids], dtype=np.int64)
        self.X = np.array([[g.vertices[v] for v in row] for row in self.lverts])
        self.jac, self.df, self.xyz = hex_geometry(self.X, np.asarray(self.T["z"][0]))
        self._assemble()

    # ------------------------------------------------------------------ #
    def _classify(self):
        """Per local mode of a hexahedron: kind (0 vertex, 1 edge, 2 face,
        3 interior) and the indices that say where it lives."""
        nm = self.nm
        p, q, r = np.meshgrid(np.arange(nm), np.arange(nm), np.arange(nm), indexing="ij")
        p, q, r = (a.transpose(2, 1, 0).reshape(-1) for a in (p, q, r))  # index p + nm(q + nm r)
        return np.stack([p, q, r], axis=1)

    def _dirichlet_faces(self):
        g, s = self.session.geometry, self.session
        faces = set()
        for rid, comps in s.boundary_regions.items():
            conds = [bc for bc in s.boundary_conditions.get(rid, []) if bc.var == self.var]
            if not conds:
                continue
            bc = conds[0]
            if bc.kind != "D":
                raise SessionError("boundary condition %r on region %d is not supported "
                                   "(Dirichlet only)" % (bc.kind, rid))
            for c in comps:
                letter, ids = g.composites[c]
                if letter not in ("F", "Q", "T"):
                    raise SessionError("boundary composite %d does not hold faces" % c)
                for f in ids:
                    faces.add(f)
                    self._face_bc[f] = bc
        return faces

    def _assemble(self):
        g, nm = self.session.geometry, self.nm
        modes = self._classify()
        bub = modes >= 2
        kind = bub.sum(axis=1)
        self._face_bc = {}
        dir_faces = self._dirichlet_faces()
        # boundary face keys (sorted vertex ids) -> face id
        def face_verts(f):
            return tuple(sorted({v for e in g.faces[f][1] for v in g.edges[e]}))
        dir_keys = {face_verts(f): f for f in dir_faces}
        nb = nm - 2
        entities = {}  # key -> (kind, size)
        refs = []  # per element, per local mode: (entity key, offset, sign)
        for el in range(self.nelmt):
            V = self.lverts[el]
            row = []
            for m in range(self.nc):
                idx = modes[m]
                k = kind[m]
                if k == 0:
                    key = ("v", int(V[HEX_CORNER[tuple(idx)]]))
                    row.append((key, 0, 1.0))
                elif k == 1:
                    d = int(np.nonzero(bub[m])[0][0])
                    lo, hi = list(idx), list(idx)
                    lo[d], hi[d] = 0, 1
                    ga, gb = int(V[HEX_CORNER[tuple(lo)]]), int(V[HEX_CORNER[tuple(hi)]])
                    key = ("e", min(ga, gb), max(ga, gb))
                    mode = int(idx[d])
                    sign = (-1.0) ** mode if ga > gb else 1.0
                    row.append((key, mode - 2, sign))
                elif k == 2:
                    d1, d2 = (int(v) for v in np.nonzero(bub[m])[0])

                    def corner(a1, a2):
                        c = list(idx)
                        c[d1], c[d2] = a1, a2
                        return int(V[HEX_CORNER[tuple(c)]])
                    cids = {(0, 0): corner(0, 0), (1, 0): corner(1, 0), (0, 1): corner(0, 1),
                            (1, 1): corner(1, 1)}
                    key = ("f",) + tuple(sorted(cids.values()))
                    (aO, bO) = min(cids, key=lambda c: cids[c])
                    n1 = cids[(1 - aO, bO)]  # neighbour along element axis 1
                    n2 = cids[(aO, 1 - bO)]  # neighbour along element axis 2
                    s1 = 1 if aO == 0 else -1
                    s2 = 1 if bO == 0 else -1
                    m1, m2 = int(idx[d1]), int(idx[d2])
                    sign = float((s1 ** m1) * (s2 ** m2))
                    ca, cb = (m1, m2) if n1 < n2 else (m2, m1)
                    row.append((key, (ca - 2) * nb + (cb - 2), sign))
                else:
                    key = ("i", el)
                    off = ((int(idx[2]) - 2) * nb + (int(idx[1]) - 2)) * nb + (int(idx[0]) - 2)
                    row.append((key, off, 1.0))
                size = {0: 1, 1: nb, 2: nb * nb, 3: nb ** 3}[k]
                entities.setdefault(key, size)
            refs.append(row)
        # Dirichlet entities: the vertices, edges and faces of Dirichlet faces
        dir_ent = set()
        for fv in dir_keys:
            dir_ent.add(("f",) + fv)
        for f in dir_faces:
            for e in g.faces[f][1]:
                a, b = g.edges[e]
                dir_ent.add(("e", min(a, b), max(a, b)))
                dir_ent.add(("v", a))
                dir_ent.add(("v", b))
        order = {"v": 0, "e": 1, "f": 2, "i": 3}
        keys = sorted(entities, key=lambda k: (k not in dir_ent, order[k[0]], k[1:]))
        base, n = {}, 0
        ndir = 0
        for k in keys:
            base[k] = n
            n += entities[k]
            if k in dir_ent:
                ndir = n
        self.nglob, self.ndir = n, ndir
        gmap = np.empty(self.nelmt * self.nc, dtype=np.int32)
        sign = np.empty(self.nelmt * self.nc)
        for el, row in enumerate(refs):
            for m, (key, off, sg) in enumerate(row):
                gmap[el * self.nc + m] = base[key] + off
                sign[el * self.nc + m] = sg
        self.gmap, self.sign = gmap, sign
        self._base, self._entities = base, entities
        self._dir_ent = dir_ent
        self._dir_keys = dir_keys

    # ------------------------------------------------------------------ #
    def dirichlet_values(self, time=0.0):
        """Global Dirichlet coefficients (ndir,) by the boundary-constrained
        projection of the boundary values on each Dirichlet face."""
        g = self.session.geometry
        B, w, z = _modA(self.T)
        nm, nb = self.nm, self.nm - 2
        out = np.zeros(self.ndir)
        P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
        bc_of = {}
        for fv, f in self._dir_keys.items():
            bc_of[fv] = self._face_bc[f]
        # vertices and edges take the condition of one face that holds them
        ent_bc = {}
        for fv, bc in bc_of.items():
            for v in fv:
                ent_bc.setdefault(("v", v), bc)
        for f, bc in self._face_bc.items():
            for e in g.faces[f][1]:
                a, b = g.edges[e]
                ent_bc.setdefault(("e", min(a, b), max(a, b)), bc)
        vals = {}
        for key, bc in ent_bc.items():
            if key[0] == "v":
                x = P(key[1])
                out[self._base[key]] = bc.value.evaluate(x[0], x[1], x[2], time)
                vals[key] = out[self._base[key]]
        # edges: 1-D constrained projection along lo -> hi
        M1 = (B[2:] * w) @ B[2:].T
        for key, bc in ent_bc.items():
            if key[0] != "e":
                continue
            xa, xb = P(key[1]), P(key[2])
            x = np.outer(0.5 * (1 - z), xa) + np.outer(0.5 * (1 + z), xb)
            f = bc.value.evaluate(x[:, 0], x[:, 1], x[:, 2], time)
            c0, c1 = f[0], f[-1]
            rem = f - c0 * B[0] - c1 * B[1]
            # the edge Jacobian (length / 2) scales both sides alike
            c = np.linalg.solve(M1, (B[2:] * w) @ rem) if nb > 0 else np.zeros(0)
            o = self._base[key]
            out[o:o + nb] = c
        # faces: 2-D constrained projection in the canonical face frame
        for fv, bc in bc_of.items():
            key = ("f",) + fv
            f = self._dir_keys[fv]
            cyc = self._face_cycle(f)
            i0 = int(np.argmin(cyc))
            O = cyc[i0]
            nA, nB = cyc[(i0 + 1) % 4], cyc[(i0 - 1) % 4]
            if nA > nB:
                nA, nB = nB, nA
            AB = cyc[(i0 + 2) % 4]
            XO, XA, XB, XAB = P(O), P(nA), P(nB), P(AB)
            za, zb = np.meshgrid(z, z, indexing="ij")  # [a, b]
            Na = [0.5 * (1 - za), 0.5 * (1 + za)]
            Nb = [0.5 * (1 - zb), 0.5 * (1 + zb)]
            x = (Na[0] * Nb[0])[..., None] * XO + (Na[1] * Nb[0])[..., None] * XA + \
                (Na[0] * Nb[1])[..., None] * XB + (Na[1] * Nb[1])[..., None] * XAB
            dxa = (0.5 * Nb[0])[..., None] * (XA - XO) + (0.5 * Nb[1])[..., None] * (XAB - XB)
            dxb = (0.5 * Na[0])[..., None] * (XB - XO) + (0.5 * Na[1])[..., None] * (XAB - XA)
            J = np.linalg.norm(np.cross(dxa, dxb), axis=-1)
            vals_f = bc.value.evaluate(x[..., 0], x[..., 1], x[..., 2], time)
            # boundary part: vertex modes, then the four edges' bubbles
            ub = (vals[("v", O)] * np.outer(B[0], B[0]) + vals[("v", nA)] * np.outer(B[1], B[0])
                  + vals[("v", nB)] * np.outer(B[0], B[1]) + vals[("v", AB)] * np.outer(B[1], B[1]))

            def edge_coeffs(a, b):
                k = ("e", min(a, b), max(a, b))
                c = out[self._base[k]:self._base[k] + nb].copy()
                if a > b:  # face direction runs against the edge's numbering
                    c *= (-1.0) ** np.arange(2, nm)
                return c
            for (a, b, side, along) in ((O, nA, 0, "a"), (nB, AB, 1, "a"), (O, nB, 0, "b"),
                                        (nA, AB, 1, "b")):
                c = edge_coeffs(a, b)
                prof = c @ B[2:]  # bubble sum along the edge, (nq,)
                if along == "a":
                    ub = ub + np.outer(prof, B[side])
                else:
                    ub = ub + np.outer(B[side], prof)
            W = np.outer(w, w) * J
            Bi = B[2:]
            rhs = np.einsum("ai,bj,ij->ab", Bi, Bi, W * (vals_f - ub)).reshape(-1)
            M2 = np.einsum("ai,ci,bj,dj,ij->abcd", Bi, Bi, Bi, Bi, W).reshape(nb * nb, nb * nb)
            c = np.linalg.solve(M2, rhs) if nb > 0 else np.zeros(0)
            o = self._base[key]
            out[o:o + nb * nb] = c
        return out

    def _face_cycle(self, f):
        """The 4 global vertex ids of face f in cyclic order."""
        g = self.session.geometry
        es = [g.edges[e] for e in g.faces[f][1]]
        cyc = [es[0][0], es[0][1]]
        while len(cyc) < 4:
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

    def dirichlet_local(self, time=0.0):
        """Local coefficient vector holding the Dirichlet values (zeros
        elsewhere), the x_loc a solve takes for the lifting."""
        dv = self.dirichlet_values(time)
        x = np.zeros(self.nelmt * self.nc)
        mask = self.gmap < self.ndir
        x[mask] = self.sign[mask] * dv[self.gmap[mask]]
        return x

    def quad_weights(self):
        """W = jac * w0 w1 w2 at every quadrature point (integration weights)."""
        w = [np.asarray(v) for v in self.T["w"]]
        wq = np.einsum("k,j,i->kji", w[2], w[1], w[0]).reshape(-1)
        return self.jac * np.tile(wq, self.nelmt)
