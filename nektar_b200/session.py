"""Reader of Nektar++ XML session files: the mesh (GEOMETRY), the expansion
orders (EXPANSIONS) and the CONDITIONS a Helmholtz solve needs.

Follows the reference readers section by section:

* vertices, edges, faces, 3-D elements, composites and the domain:
  SpatialDomains/MeshGraphIOXml.cpp v_ReadVertices (:622-801), v_ReadEdges
  (:1240-1325), v_ReadFaces (:1327-1469), v_ReadElements3D (:1718-2054),
  ReadComposites (:2056-), ReadDomain (:1144-1238);
* expansions: MeshGraph::ReadExpansionInfo (MeshGraph.cpp:3102-) for the
  `TYPE="MODIFIED"` form with one NUMMODES for all directions, per domain
  composite (different composites may have different orders);
* parameters, solver info, variables, functions: SessionReader.cpp
  ReadParameters (:1785-1867), ReadSolverInfo (:1869-1941), ReadVariables
  (:2172-2250), ReadFunctions (:2252-2475);
* boundary regions and conditions: SpatialDomains/Conditions.cpp
  ReadBoundaryRegions (:228-316), ReadBoundaryConditions (:318-).

What the B200 path does not take is rejected with a clear message rather
than read wrongly: curves beyond quadratic order (edges of more than 3
points, faces of more than 3 x 3 or 6), compressed (base64) geometry blocks,
per-direction orders (NUMMODES="4,6,8"), pyramids, and expansion types
other than MODIFIED.
"""
import re
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np

from .expr import Expression, evaluate_parameters


class SessionError(ValueError):
    pass


# element letters of the GEOMETRY section (MeshGraphIOXml.cpp v_ReadElements3D)
ELEMENT_SHAPES = {"H": "hex", "R": "prism", "A": "tet", "P": "pyramid"}


@dataclass
class Geometry:
    dim: int
    space: int
    vertices: dict  # id -> (x, y, z)
    edges: dict  # id -> (v0, v1)
    faces: dict  # id -> ('Q' | 'T', [edge ids])
    elements: dict  # id -> (shape, [face ids])
    composites: dict  # id -> (letter, [ids])
    domain: list  # composite ids
    curved_edges: dict = field(default_factory=dict)  # edge id -> (npts, 3) curve points
    curved_faces: dict = field(default_factory=dict)  # face id -> (npts, 3) face points


@dataclass
class BoundaryCondition:
    kind: str  # 'D' Dirichlet, 'N' Neumann, 'R' Robin
    var: str
    value: Expression
    primcoeff: Expression = None  # Robin


@dataclass
class Session:
    name: str
    geometry: Geometry
    nummodes: dict  # composite id -> NUMMODES
    exp_type: str
    parameters: dict
    solver_info: dict
    variables: list
    boundary_regions: dict  # region id -> [composite ids]
    boundary_conditions: dict  # region id -> [BoundaryCondition]
    functions: dict = field(default_factory=dict)  # name -> {var: Expression}

    def function(self, name, var=None):
        f = self.functions.get(name)
        if not f:
            return None
        return f.get(var or self.variables[0], next(iter(f.values())))


def parse_id_list(text):
    """'0-3,7,9-10' -> [0, 1, 2, 3, 7, 9, 10] (ParseUtils::GenerateSeqVector)."""
    out = []
    for part in text.replace(" ", "").split(","):
        if not part:
            continue
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        else:
            out.append(int(part))
    return out


def parse_composite_refs(text):
    """'H[0-7]' or 'F[1,2] F[4]' -> [(letter, [ids]), ...]."""
    refs = re.findall(r"([A-Za-z])\s*\[([^\]]*)\]", text)
    if not refs:
        raise SessionError("cannot parse composite reference %r" % text)
    return [(letter, parse_id_list(ids)) for letter, ids in refs]


def _ints(text):
    return [int(v) for v in text.split()]


def _read_geometry(root):
    g = root.find("GEOMETRY")
    if g is None:
        raise SessionError("no GEOMETRY section")
    dim, space = int(g.get("DIM", 3)), int(g.get("SPACE", 3))
    curved, curved_faces = {}, {}
    cnode = g.find("CURVED")
    for c in (list(cnode) if cnode is not None else []):
        # MeshGraphIOXml::v_ReadCurves: edges and faces with their points;
        # quadratic curves only (an edge's two vertices and midpoint; a
        # quadrilateral's 3 x 3 points, a triangle's 6)
        npts, ptype = int(c.get("NUMPOINTS")), c.get("TYPE")
        vals = np.array([float(v) for v in c.text.split()], dtype=np.float64)
        if c.tag == "F":
            if npts not in (6, 9) or ptype not in ("PolyEvenlySpaced", "GaussLobattoLegendre"):
                raise SessionError("curved face %s: %d %s points (quadratic curves only)"
                                   % (c.get("FACEID"), npts, ptype))
            curved_faces[int(c.get("FACEID"))] = vals.reshape(npts, 3)
            continue
        if c.tag != "E":
            raise SessionError("curved %s records are not supported" % c.tag)
        if npts != 3 or ptype not in ("PolyEvenlySpaced", "GaussLobattoLegendre"):
            raise SessionError("curved edge %s: %d %s points (quadratic curves only)"
                               % (c.get("EDGEID"), npts, ptype))
        curved[int(c.get("EDGEID"))] = vals.reshape(npts, 3)
    for sec in ("VERTEX", "EDGE", "FACE", "ELEMENT"):
        node = g.find(sec)
        if node is not None and node.get("COMPRESSED"):
            raise SessionError("compressed %s blocks are not supported" % sec)
    vnode = g.find("VERTEX")
    scale = [1.0, 1.0, 1.0]
    move = [0.0, 0.0, 0.0]
    for k, ax in enumerate("XYZ"):
        if vnode.get(ax + "SCALE"):
            scale[k] = float(Expression(vnode.get(ax + "SCALE")).evaluate())
        if vnode.get(ax + "MOVE"):
            move[k] = float(Expression(vnode.get(ax + "MOVE")).evaluate())
    vertices = {}
    for v in vnode.findall("V"):
        xyz = [float(s) for s in v.text.split()]
        vertices[int(v.get("ID"))] = tuple(xyz[k] * scale[k] + move[k] for k in range(3))
    edges = {}
    enode = g.find("EDGE")
    if enode is not None:
        for e in enode.findall("E"):
            a, b = _ints(e.text)
            edges[int(e.get("ID"))] = (a, b)
    faces = {}
    fnode = g.find("FACE")
    if fnode is not None:
        for f in fnode:
            if f.tag not in ("Q", "T"):
                continue
            ids = _ints(f.text)
            if len(ids) != (4 if f.tag == "Q" else 3):
                raise SessionError("face %s has %d edges" % (f.get("ID"), len(ids)))
            faces[int(f.get("ID"))] = (f.tag, ids)
    elements = {}
    for el in g.find("ELEMENT"):
        shape = ELEMENT_SHAPES.get(el.tag)
        if shape is None:
            raise SessionError("element type %r is not a 3-D element" % el.tag)
        if shape == "pyramid":
            raise SessionError("pyramids are not supported")
        elements[int(el.get("ID"))] = (shape, _ints(el.text))
    composites = {}
    cnode = g.find("COMPOSITE")
    for c in cnode.findall("C"):
        refs = parse_composite_refs(c.text)
        letters = {r[0] for r in refs}
        if len(letters) != 1:
            # a composite holds one kind of entity (faces, or elements)
            kinds = {"F" if l in "QTF" else "E" for l in letters}
            if len(kinds) != 1:
                raise SessionError("composite %s mixes faces and elements" % c.get("ID"))
        ids = [i for _, lst in refs for i in lst]
        composites[int(c.get("ID"))] = (refs[0][0], ids)
    dnode = g.find("DOMAIN")
    domain = [i for _, lst in parse_composite_refs(dnode.text) for i in lst]
    for e, pts in curved.items():
        ends = {tuple(np.round(pts[0], 12)), tuple(np.round(pts[-1], 12))}
        want = {tuple(np.round(np.asarray(vertices[v], dtype=np.float64), 12)) for v in edges[e]}
        if ends != want:
            raise SessionError("curved edge %d does not end at its vertices" % e)
    for f, pts in curved_faces.items():
        if f not in faces:
            raise SessionError("curved face %d is no face of the mesh" % f)
        kind, fe = faces[f]
        if (kind == "Q") != (len(pts) == 9):
            raise SessionError("curved face %d: %d points for a %s" % (
                f, len(pts), "quadrilateral" if kind == "Q" else "triangle"))
        want = {tuple(np.round(np.asarray(vertices[v], dtype=np.float64), 12))
                for e in fe for v in edges[e]}
        # a quadrilateral's points in tensor order: corners 0, 2, 6, 8
        got = {tuple(np.round(pts[i], 12)) for i in ((0, 2, 6, 8) if kind == "Q" else
                                                       range(len(pts)))}
        if not want <= got or (kind == "Q" and got != want):
            raise SessionError("curved face %d does not have its vertices as corners" % f)
    return Geometry(dim, space, vertices, edges, faces, elements, composites, domain, curved,
                    curved_faces)


# the bases and points TYPE="MODIFIED" gives each shape at nm modes
# (SpatialDomains/MeshGraph.cpp:1709-1750): basis types, point types and point
# counts (nm + 1 GLL points, nm Gauss-Radau points in collapsed directions)
_MODIFIED = {
    "H": (("Modified_A",) * 3, ("GaussLobattoLegendre",) * 3, (1, 1, 1)),
    "R": (("Modified_A", "Modified_A", "Modified_B"),
          ("GaussLobattoLegendre", "GaussLobattoLegendre", "GaussRadauMAlpha1Beta0"), (1, 1, 0)),
    "A": (("Modified_A", "Modified_B", "Modified_C"),
          ("GaussLobattoLegendre", "GaussRadauMAlpha1Beta0", "GaussRadauMAlpha2Beta0"),
          (1, 0, 0)),
}


def _explicit_order(e, letters):
    """The order of an explicit expansion (BASISTYPE, NUMMODES, POINTSTYPE,
    NUMPOINTS per direction) when it is the one TYPE="MODIFIED" gives the
    composite's shapes at one order in all directions; SessionError naming
    what differs otherwise."""
    def parts(key):
        v = e.get(key)
        if v is None:
            raise SessionError("explicit expansion without %s" % key)
        return [x.strip() for x in v.split(",")]
    nms = [int(x) for x in parts("NUMMODES")]
    nqs = [int(x) for x in parts("NUMPOINTS")]
    if len(set(nms)) != 1:
        raise SessionError("per-direction orders NUMMODES=%s are not supported" %
                           ",".join(map(str, nms)))
    nm = nms[0]
    bts, pts = parts("BASISTYPE"), parts("POINTSTYPE")
    for letter in letters:
        if letter not in _MODIFIED:
            raise SessionError("no expansion for element type %r" % letter)
        want_b, want_p, extra = _MODIFIED[letter]
        want_q = [nm + x for x in extra]
        if len(bts) == 1:
            bts = bts * 3
        if len(pts) == 1:
            pts = pts * 3
        if len(nqs) == 1:
            nqs = nqs * 3
        if (tuple(bts), tuple(pts), list(nqs)) != (want_b, want_p, want_q):
            raise SessionError("explicit expansion %s / %s / %s is not the standard modified "
                               "expansion of its elements (%s / %s / %s)" % (
                                   ",".join(bts), ",".join(pts), ",".join(map(str, nqs)),
                                   ",".join(want_b), ",".join(want_p), ",".join(map(str, want_q))))
    return nm


def _read_expansions(root, composites):
    node = root.find("EXPANSIONS")
    if node is None:
        raise SessionError("no EXPANSIONS section")
    nummodes, etype = {}, None
    for e in node.findall("E"):
        refs = parse_composite_refs(e.get("COMPOSITE"))
        t = e.get("TYPE")
        if t is None:
            letters = {composites[c][0] for _, ids in refs for c in ids if c in composites}
            nm = _explicit_order(e, letters)
        else:
            if t.upper() != "MODIFIED":
                raise SessionError("expansion type %r is not supported (MODIFIED only)" % t)
            nmt = e.get("NUMMODES").replace(" ", "")
            if "," in nmt:
                raise SessionError("per-direction orders NUMMODES=%r are not supported" % nmt)
            nm = int(nmt)
        for _, ids in refs:
            for c in ids:
                nummodes[c] = nm
        etype = "MODIFIED"
    return nummodes, etype


def _read_conditions(root):
    cond = root.find("CONDITIONS")
    pairs, solver_info, variables = [], {}, []
    regions, bcs, funcs_raw = {}, {}, {}
    if cond is None:
        return evaluate_parameters(pairs), solver_info, variables, regions, bcs, funcs_raw
    pnode = cond.find("PARAMETERS")
    if pnode is not None:
        for p in pnode.findall("P"):
            lhs, rhs = p.text.split("=", 1)
            pairs.append((lhs.strip(), rhs.strip()))
    snode = cond.find("SOLVERINFO")
    if snode is not None:
        for i in snode.findall("I"):
            solver_info[i.get("PROPERTY")] = i.get("VALUE")
    vnode = cond.find("VARIABLES")
    if vnode is not None:
        variables = [v.text.strip() for v in sorted(vnode.findall("V"), key=lambda v: int(v.get("ID")))]
    rnode = cond.find("BOUNDARYREGIONS")
    if rnode is not None:
        for b in rnode.findall("B"):
            regions[int(b.get("ID"))] = [i for _, lst in parse_composite_refs(b.text) for i in lst]
    bnode = cond.find("BOUNDARYCONDITIONS")
    if bnode is not None:
        for r in bnode.findall("REGION"):
            bcs[int(r.get("REF"))] = [(c.tag, c.get("VAR"), c.get("VALUE"), c.get("PRIMCOEFF"))
                                      for c in r]
    for f in cond.findall("FUNCTION"):
        entries = {}
        for e in f.findall("E"):
            if e.get("VALUE") is None:
                raise SessionError("function %s: only VALUE expressions are supported"
                                   % f.get("NAME"))
            for v in e.get("VAR").split(","):
                entries[v.strip()] = e.get("VALUE")
        funcs_raw[f.get("NAME")] = entries
    return evaluate_parameters(pairs), solver_info, variables, regions, bcs, funcs_raw


def read_session(path_or_text):
    """Read a session from a file path or an XML string."""
    text = path_or_text
    name = "session"
    if not path_or_text.lstrip().startswith("<"):
        with open(path_or_text) as fh:
            text = fh.read()
        name = re.sub(r"\.xml$", "", path_or_text.split("/")[-1])
    root = ET.fromstring(text)
    if root.tag != "NEKTAR":
        raise SessionError("root element is %r, not NEKTAR" % root.tag)
    geom = _read_geometry(root)
    nummodes, etype = _read_expansions(root, geom.composites)
    params, solver_info, variables, regions, bcs_raw, funcs_raw = _read_conditions(root)
    bcs = {}
    for rid, lst in bcs_raw.items():
        out = []
        for kind, var, value, prim in lst:
            if kind not in ("D", "N", "R"):
                raise SessionError("boundary condition %r is not supported" % kind)
            out.append(BoundaryCondition(kind, var, Expression(value, params),
                                         Expression(prim, params) if prim else None))
        bcs[rid] = out
    funcs = {n: {v: Expression(t, params) for v, t in d.items()} for n, d in funcs_raw.items()}
    return Session(name, geom, nummodes, etype, params, solver_info, variables, regions, bcs,
                   funcs)


# ---------------------------------------------------------------------------
# writer (meshes generated here, in the same format the reader takes)
# ---------------------------------------------------------------------------

def _seq(ids):
    """[0, 1, 2, 5] -> '0-2,5' (ParseUtils::GenerateSeqString)."""
    ids = sorted(ids)
    out, i = [], 0
    while i < len(ids):
        j = i
        while j + 1 < len(ids) and ids[j + 1] == ids[j] + 1:
            j += 1
        out.append(str(ids[i]) if i == j else "%d-%d" % (ids[i], ids[j]))
        i = j + 1
    return ",".join(out)


def _cube_rotations():
    """The 24 proper rotations of the cube as signed permutation matrices."""
    import itertools
    out = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1, -1), repeat=3):
            R = np.zeros((3, 3), dtype=int)
            for r, c in enumerate(perm):
                R[r, c] = signs[r]
            if round(np.linalg.det(R)) == 1:
                out.append(R)
    return out


def write_hex_box_session(n, nummodes, lam, dirichlet, forcing, exact, lengths=(1.0, 1.0, 1.0),
                          shuffle_seed=None):
    """XML text of a session on the box [0,Lx]x[0,Ly]x[0,Lz] cut into n^3
    hexes, Dirichlet data on all six sides. Faces are listed bottom, four
    sides, top per element, the order HexGeom::SetUpLocalEdges expects.
    With shuffle_seed every element's local frame is one of the 24 proper
    rotations of the cube and every edge lists its vertices in a random
    order (seeded), so that neighbouring elements meet with all relative
    orientations of their edges and faces."""
    rng = np.random.default_rng(shuffle_seed) if shuffle_seed is not None else None
    rots = _cube_rotations()
    corner_xi = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1),
                 (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    N = n + 1
    vid = lambda i, j, k: (k * N + j) * N + i  # noqa: E731
    lines = ['<?xml version="1.0" encoding="utf-8" ?>', "<NEKTAR>",
             '  <GEOMETRY DIM="3" SPACE="3">', "    <VERTEX>"]
    for k in range(N):
        for j in range(N):
            for i in range(N):
                lines.append('      <V ID="%d">%.17g %.17g %.17g</V>' % (
                    vid(i, j, k), lengths[0] * i / n, lengths[1] * j / n, lengths[2] * k / n))
    lines.append("    </VERTEX>")
    edges, emap = [], {}

    def edge(a, b):
        key = (min(a, b), max(a, b))
        if key not in emap:
            emap[key] = len(edges)
            edges.append((b, a) if rng is not None and rng.integers(2) else (a, b))
        return emap[key]

    faces, fmap = [], {}

    def face(cyc):
        key = tuple(sorted(cyc))
        if key not in fmap:
            fmap[key] = len(faces)
            faces.append([edge(cyc[m], cyc[(m + 1) % 4]) for m in range(4)])
        return fmap[key]

    elems, bnd = [], {s: [] for s in range(6)}
    for k in range(n):
        for j in range(n):
            for i in range(n):
                v = [vid(i, j, k), vid(i + 1, j, k), vid(i + 1, j + 1, k), vid(i, j + 1, k),
                     vid(i, j, k + 1), vid(i + 1, j, k + 1), vid(i + 1, j + 1, k + 1),
                     vid(i, j + 1, k + 1)]
                if rng is not None:
                    # local corner c sits where the rotation R takes it
                    R = rots[int(rng.integers(len(rots)))]
                    where = {xi: m for m, xi in enumerate(corner_xi)}
                    v = [v[where[tuple(int(t) for t in R @ np.array(xi))]] for xi in corner_xi]
                f = [face([v[0], v[1], v[2], v[3]]), face([v[0], v[1], v[5], v[4]]),
                     face([v[1], v[2], v[6], v[5]]), face([v[3], v[2], v[6], v[7]]),
                     face([v[0], v[3], v[7], v[4]]), face([v[4], v[5], v[6], v[7]])]
                elems.append(f)
                # boundary faces by position: a face on a side of the box has
                # all its vertices there
                for fid in f:
                    vs = {x for ed in faces[fid] for x in edges[ed]}
                    ijk = [((x % N), (x // N) % N, x // (N * N)) for x in vs]
                    for side, (ax, val) in enumerate(((2, 0), (1, 0), (0, n), (1, n), (0, 0),
                                                      (2, n))):
                        if all(t[ax] == val for t in ijk) and fid not in bnd[side]:
                            bnd[side].append(fid)
    lines.append("    <EDGE>")
    lines += ['      <E ID="%d"> %d %d </E>' % (e, a, b) for e, (a, b) in enumerate(edges)]
    lines.append("    </EDGE>")
    lines.append("    <FACE>")
    lines += ['      <Q ID="%d"> %s </Q>' % (q, " ".join(map(str, es))) for q, es in enumerate(faces)]
    lines.append("    </FACE>")
    lines.append("    <ELEMENT>")
    lines += ['      <H ID="%d"> %s </H>' % (e, " ".join(map(str, fs))) for e, fs in enumerate(elems)]
    lines.append("    </ELEMENT>")
    lines.append("    <COMPOSITE>")
    lines.append('      <C ID="0"> H[%s] </C>' % _seq(range(len(elems))))
    for s in range(6):
        lines.append('      <C ID="%d"> F[%s] </C>' % (s + 1, _seq(bnd[s])))
    lines += ["    </COMPOSITE>", "    <DOMAIN> C[0] </DOMAIN>", "  </GEOMETRY>",
              "  <EXPANSIONS>",
              '    <E COMPOSITE="C[0]" NUMMODES="%d" FIELDS="u" TYPE="MODIFIED" />' % nummodes,
              "  </EXPANSIONS>", "  <CONDITIONS>", "    <PARAMETERS>",
              "      <P> Lambda = %.17g </P>" % lam, "    </PARAMETERS>",
              '    <VARIABLES> <V ID="0"> u </V> </VARIABLES>',
              '    <BOUNDARYREGIONS> <B ID="0"> C[1-6] </B> </BOUNDARYREGIONS>',
              "    <BOUNDARYCONDITIONS>", '      <REGION REF="0">',
              '        <D VAR="u" VALUE="%s" />' % dirichlet, "      </REGION>",
              "    </BOUNDARYCONDITIONS>",
              '    <FUNCTION NAME="Forcing"> <E VAR="u" VALUE="%s" /> </FUNCTION>' % forcing,
              '    <FUNCTION NAME="ExactSolution"> <E VAR="u" VALUE="%s" /> </FUNCTION>' % exact,
              "  </CONDITIONS>", "</NEKTAR>"]
    return "\n".join(lines) + "\n"


def with_orders(xml_text, orders, seed=0):
    """The session xml_text with its elements spread over len(orders)
    domain composites (seeded, every composite of every element type
    non-empty where there are enough elements), composite k expanded with
    orders[k] modes: a variable-order session as the reference's *_VarP
    tests have them."""
    import xml.etree.ElementTree as ET
    root = ET.fromstring(xml_text)
    geom = root.find("GEOMETRY")
    comp = geom.find("COMPOSITE")
    dom_ids = parse_id_list(geom.find("DOMAIN").text.strip()[2:-1])
    rng = np.random.default_rng(seed)
    new = {}
    for c in list(comp):
        if int(c.get("ID")) not in dom_ids:
            continue
        txt = c.text.strip()
        letter, ids = txt[0], parse_id_list(txt[2:-1])
        comp.remove(c)
        perm = rng.permutation(len(ids))
        for k in range(len(orders)):
            part = sorted(ids[i] for i in perm[k::len(orders)])
            if part:
                new.setdefault(k, []).append("%s[%s]" % (letter, _seq(part)))
    cids = []
    for k, parts in sorted(new.items()):
        cid = 100 + k
        e = ET.SubElement(comp, "C", ID=str(cid))
        e.text = " " + " ".join(parts) + " "
        cids.append(cid)
    geom.find("DOMAIN").text = " C[%s] " % ",".join(map(str, cids))
    exps = root.find("EXPANSIONS")
    for e in list(exps):
        exps.remove(e)
    for k, cid in zip(sorted(new), cids):
        ET.SubElement(exps, "E", COMPOSITE="C[%d]" % cid, NUMMODES=str(orders[k]), FIELDS="u",
                      TYPE="MODIFIED")
    return ET.tostring(root, encoding="unicode")


# Conditions of the reference's Helmholtz3D_Hex_AllBCs session on the box
# writers' six sides (C[1] z=0, C[2] y=0, C[3] x=1, C[4] y=1, C[5] x=0,
# C[6] z=1) for u = sin(PI/2 x) sin(PI/2 y) sin(PI/2 z): Dirichlet, Neumann
# (the outward normal derivative) and Robin (du/dn + a u) data
ALL_BCS = [
    ([1, 5], "D", "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)", None),
    ([2], "N", "-sin(PI/2*x)*cos(PI/2*y)*sin(PI/2*z)*PI/2", None),
    ([3], "R", "cos(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)*PI/2+2*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)",
     "2"),
    ([4], "R", "sin(PI/2*x)*cos(PI/2*y)*sin(PI/2*z)*PI/2+3*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)",
     "3"),
    ([6], "N", "sin(PI/2*x)*sin(PI/2*y)*cos(PI/2*z)*PI/2", None),
]


def with_conditions(xml_text, regions):
    """The session xml_text with its boundary regions and conditions
    replaced: regions is a list of (composite ids, kind 'D' / 'N' / 'R',
    VALUE, PRIMCOEFF or None), one boundary region each."""
    import xml.etree.ElementTree as ET
    root = ET.fromstring(xml_text)
    cond = root.find("CONDITIONS")
    for tag in ("BOUNDARYREGIONS", "BOUNDARYCONDITIONS"):
        old = cond.find(tag)
        if old is not None:
            cond.remove(old)
    br = ET.SubElement(cond, "BOUNDARYREGIONS")
    bc = ET.SubElement(cond, "BOUNDARYCONDITIONS")
    for rid, (comps, kind, value, prim) in enumerate(regions):
        b = ET.SubElement(br, "B", ID=str(rid))
        b.text = " C[%s] " % _seq(sorted(comps))
        r = ET.SubElement(bc, "REGION", REF=str(rid))
        e = ET.SubElement(r, kind, VAR="u", VALUE=value)
        if prim is not None:
            e.set("PRIMCOEFF", prim)
    return ET.tostring(root, encoding="unicode")


def write_box_session(shape, n, nummodes, lam, dirichlet, forcing, exact, shuffle_seed=None):
    """XML text of a session on the unit cube cut into n^3 cells, each a
    hexahedron, two prisms (triangles in the x-z plane, extruded along y) or
    six tetrahedra (the cell split along its main diagonal), with Dirichlet
    data on all six sides. Elements list their faces in the order of the
    reference's geometry classes; every tetrahedron has its vertices in
    increasing id (v0 and v1 swapped where that would invert it), so
    neighbouring triangles collapse towards the same vertex and each face's
    first edge is the one TetGeom expects; a triangle lists its edges
    origin -> end of axis a -> apex of the element that first uses it, so
    that its own frame (TriGeom: vertex j starts edge j) collapses towards the
    element's apex. shuffle_seed (hexahedra:
    random frames, see write_hex_box_session; prisms and tetrahedra: random
    edge directions and quadrilateral edge lists)."""
    if shape == "hex":
        return write_hex_box_session(n, nummodes, lam, dirichlet, forcing, exact,
                                     shuffle_seed=shuffle_seed)
    # "hexprism": hexahedra for x < 1/2, prisms for x > 1/2 (two collections)
    rng = np.random.default_rng(shuffle_seed) if shuffle_seed is not None else None
    N = n + 1
    vid = lambda i, j, k: (k * N + j) * N + i  # noqa: E731
    coords = {vid(i, j, k): (i / n, j / n, k / n) for k in range(N) for j in range(N)
              for i in range(N)}
    edges, emap, faces, fmap = [], {}, [], {}

    def edge(a, b):
        key = (min(a, b), max(a, b))
        if key not in emap:
            emap[key] = len(edges)
            edges.append((b, a) if rng is not None and rng.integers(2) else (a, b))
        return emap[key]

    def face(cyc):
        key = tuple(sorted(cyc))
        if key not in fmap:
            if len(cyc) == 3:
                # (origin, end of axis a, apex): the triangle's own frame has
                # its vertex 2 where the element collapses it
                es = [edge(cyc[0], cyc[1]), edge(cyc[1], cyc[2]), edge(cyc[2], cyc[0])]
            else:
                es = [edge(cyc[m], cyc[(m + 1) % 4]) for m in range(4)]
                if rng is not None:
                    r = int(rng.integers(4))
                    es = es[r:] + es[:r]
            fmap[key] = len(faces)
            faces.append(("T" if len(cyc) == 3 else "Q", es))
        return fmap[key]

    elems = []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                c = lambda a, b, cc: vid(i + a, j + b, k + cc)  # noqa: E731
                if shape == "hexprism" and 2 * i < n:
                    v = [c(0, 0, 0), c(1, 0, 0), c(1, 1, 0), c(0, 1, 0), c(0, 0, 1), c(1, 0, 1),
                         c(1, 1, 1), c(0, 1, 1)]
                    elems.append(("H", [face([v[0], v[1], v[2], v[3]]), face([v[0], v[1], v[5], v[4]]),
                                        face([v[1], v[2], v[6], v[5]]), face([v[3], v[2], v[6], v[7]]),
                                        face([v[0], v[3], v[7], v[4]]), face([v[4], v[5], v[6], v[7]])]))
                elif shape in ("prism", "hexprism"):
                    for v in ([c(0, 0, 0), c(1, 0, 0), c(1, 1, 0), c(0, 1, 0), c(0, 0, 1), c(0, 1, 1)],
                              [c(1, 0, 1), c(0, 0, 1), c(0, 1, 1), c(1, 1, 1), c(1, 0, 0), c(1, 1, 0)]):
                        elems.append(("R", [face([v[0], v[1], v[2], v[3]]), face([v[0], v[1], v[4]]),
                                            face([v[1], v[2], v[5], v[4]]), face([v[3], v[2], v[5]]),
                                            face([v[0], v[3], v[5], v[4]])]))
                else:
                    import itertools
                    for perm in itertools.permutations(range(3)):
                        pos = [0, 0, 0]
                        path = [c(0, 0, 0)]
                        for ax in perm[:2]:
                            pos[ax] = 1
                            path.append(c(*pos))
                        path.append(c(1, 1, 1))
                        v = sorted(path)
                        X = np.array([coords[x] for x in v])
                        if np.linalg.det(np.array([X[1] - X[0], X[2] - X[0], X[3] - X[0]])) < 0:
                            v[0], v[1] = v[1], v[0]
                        elems.append(("A", [face([v[0], v[1], v[2]]), face([v[0], v[1], v[3]]),
                                            face([v[1], v[2], v[3]]), face([v[0], v[2], v[3]])]))
    bnd = {s_: [] for s_ in range(6)}
    for fid, (kind, es) in enumerate(faces):
        vs = {x for ed in es for x in edges[ed]}
        ijk = [(x % N, (x // N) % N, x // (N * N)) for x in vs]
        for side, (ax, val) in enumerate(((2, 0), (1, 0), (0, n), (1, n), (0, 0), (2, n))):
            if all(t[ax] == val for t in ijk):
                bnd[side].append(fid)
    lines = ['<?xml version="1.0" encoding="utf-8" ?>', "<NEKTAR>",
             '  <GEOMETRY DIM="3" SPACE="3">', "    <VERTEX>"]
    lines += ['      <V ID="%d">%.17g %.17g %.17g</V>' % ((v,) + coords[v]) for v in sorted(coords)]
    lines += ["    </VERTEX>", "    <EDGE>"]
    lines += ['      <E ID="%d"> %d %d </E>' % (e, a, b) for e, (a, b) in enumerate(edges)]
    lines += ["    </EDGE>", "    <FACE>"]
    lines += ['      <%s ID="%d"> %s </%s>' % (kd, f, " ".join(map(str, es)), kd)
              for f, (kd, es) in enumerate(faces)]
    lines += ["    </FACE>", "    <ELEMENT>"]
    lines += ['      <%s ID="%d"> %s </%s>' % (t, e, " ".join(map(str, fs)), t)
              for e, (t, fs) in enumerate(elems)]
    # one domain composite per element type (C[0], C[7], ...), boundary sides C[1-6]
    kinds = sorted({t for t, _ in elems}, key="HRA".index)
    cids = {t: (0 if m == 0 else 6 + m) for m, t in enumerate(kinds)}
    lines += ["    </ELEMENT>", "    <COMPOSITE>"]
    lines += ['      <C ID="%d"> %s[%s] </C>' % (cids[t], t, _seq([e for e, (tt, _) in enumerate(elems)
                                                                 if tt == t])) for t in kinds]
    lines += ['      <C ID="%d"> F[%s] </C>' % (s_ + 1, _seq(bnd[s_])) for s_ in range(6)]
    dom = ",".join(str(cids[t]) for t in kinds)
    lines += ["    </COMPOSITE>", "    <DOMAIN> C[%s] </DOMAIN>" % dom, "  </GEOMETRY>",
              "  <EXPANSIONS>",
              '    <E COMPOSITE="C[%s]" NUMMODES="%d" FIELDS="u" TYPE="MODIFIED" />' % (dom, nummodes),
              "  </EXPANSIONS>", "  <CONDITIONS>", "    <PARAMETERS>",
              "      <P> Lambda = %.17g </P>" % lam, "    </PARAMETERS>",
              '    <VARIABLES> <V ID="0"> u </V> </VARIABLES>',
              '    <BOUNDARYREGIONS> <B ID="0"> C[1-6] </B> </BOUNDARYREGIONS>',
              "    <BOUNDARYCONDITIONS>", '      <REGION REF="0">',
              '        <D VAR="u" VALUE="%s" />' % dirichlet, "      </REGION>",
              "    </BOUNDARYCONDITIONS>",
              '    <FUNCTION NAME="Forcing"> <E VAR="u" VALUE="%s" /> </FUNCTION>' % forcing,
              '    <FUNCTION NAME="ExactSolution"> <E VAR="u" VALUE="%s" /> </FUNCTION>' % exact,
              "  </CONDITIONS>", "</NEKTAR>"]
    return "\n".join(lines) + "\n"
