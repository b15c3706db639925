"""Session front end on the CPU: the expression grammar, the XML reader,
hexahedral element frames, the oriented C0 assembly, and - through the
oracle - the whole discretisation against the reference's recorded errors
(library/Demos/MultiRegions/Tests/Helmholtz3D_CG_Hex.tst: L2 1.11818e-07,
Linf 5.66374e-07, tolerance 1e-12, for Helmholtz3D_Hex_P6.xml: the unit cube
cut into 2^3 hexahedra, NUMMODES 6, Lambda 1, u = sin(pi x/2) sin(pi y/2)
sin(pi z/2) on the boundary)."""
import os
from collections import defaultdict

import numpy as np
import pytest

from nektar_b200.expr import Expression, ExpressionError, evaluate_parameters
from nektar_b200.meshgraph import SessionMesh
from nektar_b200.session import SessionError, read_session, write_hex_box_session
from oracle import oracle as O
from tests.helpers import ref_path
from tests.session_oracle import oracle_helm_solve

U = "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
F = "-(Lambda + 3*PI*PI/4)*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
HEX_L2, HEX_LINF = 1.11818e-07, 5.66374e-07  # Helmholtz3D_CG_Hex.tst
REF_HEX = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Hex_P6.xml")


def test_expression_grammar():
    assert Expression("-x^2").evaluate(3.0) == -9.0  # '-' applies to the whole term
    assert Expression("2^3^2").evaluate() == 512.0  # '^' is right associative
    assert Expression("1 - -x").evaluate(2.0) == 3.0
    assert Expression("x < 1 && y >= 2 || 0").evaluate(0.5, 2.0) == 1.0
    assert Expression("fmod(7, 3) + abs(-2) + sqrt(PI_4 * 4 / PI)").evaluate() == 4.0
    v = Expression(F, {"Lambda": 2.5}).evaluate(0.2, 0.4, 0.6)
    assert np.isclose(v, -(2.5 + 3 * np.pi ** 2 / 4) * np.prod(np.sin(np.pi / 2 * np.array([.2, .4, .6]))))
    x = np.linspace(0, 1, 7)
    assert Expression("x*y").evaluate(x, 2.0).shape == (7,)
    for bad in ("2*-3", "foo + 1", "awgn(1)", "sin(1, 2)", "(1"):
        with pytest.raises(ExpressionError):
            Expression(bad).evaluate()
    assert evaluate_parameters([("A", "2"), ("B", "A^2 + PI*0")]) == {"A": 2.0, "B": 4.0}


def _session(n=2, nm=6, seed=None):
    return read_session(write_hex_box_session(n, nm, 1.0, U, F, U, shuffle_seed=seed))


def test_reader_and_mesh_counts():
    s = _session(3, 5)
    assert s.parameters["Lambda"] == 1.0 and s.variables == ["u"]
    assert len(s.geometry.elements) == 27 and len(s.geometry.vertices) == 64
    m = SessionMesh(s)
    assert (m.nglob, m.ndir) == (13 ** 3, 13 ** 3 - 11 ** 3)
    assert m.jac.shape == (27 * 216,) and m.df.shape == (9, 27 * 216)
    assert np.isclose(m.quad_weights().sum(), 1.0)  # volume of the unit cube


@pytest.mark.parametrize("seed", [None, 1, 2])
def test_assembly_is_continuous_across_all_relative_orientations(seed):
    """A random global vector scattered with the map and signs is one
    continuous function: it takes one value wherever elements share a
    quadrature point, with element frames rotated at random (seeded)."""
    m = SessionMesh(_session(3, 6, seed))
    if seed is not None:
        assert (m.sign < 0).sum() > 500  # the orientation signs are exercised
    xg = np.random.default_rng(7).uniform(-1, 1, m.nglob)
    u = O.bwdtrans("hex", m.nm, m.nq, m.nelmt, m.T["b"], m.sign * xg[m.gmap])
    vals = defaultdict(list)
    for p, v in zip(np.round(m.xyz.T, 9), u):
        vals[tuple(p)].append(v)
    assert max(max(v) - min(v) for v in vals.values()) < 1e-14


def test_dirichlet_projection_is_exact_for_polynomials():
    """A trace in the discrete space is reproduced by the boundary-constrained
    projection: quadratic data -> the lifted field equals it on the boundary."""
    s = read_session(write_hex_box_session(2, 4, 1.0, "x*x + 2*y*z - z", "0", "0", shuffle_seed=3))
    m = SessionMesh(s)
    u = O.bwdtrans("hex", m.nm, m.nq, m.nelmt, m.T["b"], m.dirichlet_local())
    x, y, z = m.xyz
    on = (np.isclose(x, 0) | np.isclose(x, 1) | np.isclose(y, 0) | np.isclose(y, 1) |
          np.isclose(z, 0) | np.isclose(z, 1))
    assert np.abs(u[on] - (x * x + 2 * y * z - z)[on]).max() < 1e-13


@pytest.mark.parametrize("seed", [None, 4])
def test_oracle_solve_reproduces_reference_record(seed):
    _, linf, l2 = oracle_helm_solve(_session(2, 6, seed))
    assert abs(l2 - HEX_L2) < 1e-12 and abs(linf - HEX_LINF) < 1e-12


@pytest.mark.skipif(not os.path.exists(REF_HEX), reason="reference tree not mounted")
def test_reference_session_file_reads_and_reproduces_its_record():
    s = read_session(REF_HEX)
    assert len(s.geometry.elements) == 8 and s.nummodes == {0: 6}
    _, linf, l2 = oracle_helm_solve(s)
    assert abs(l2 - HEX_L2) < 1e-12 and abs(linf - HEX_LINF) < 1e-12


def test_reader_rejects_what_the_path_does_not_take():
    txt = write_hex_box_session(1, 4, 1.0, U, F, U)
    with pytest.raises(SessionError):
        read_session(txt.replace('NUMMODES="4"', 'NUMMODES="4,5,6"'))
    with pytest.raises(SessionError):  # a cubic curve
        read_session(txt.replace("</GEOMETRY>", '<CURVED><E ID="0" EDGEID="0" NUMPOINTS="4" '
                                 'TYPE="PolyEvenlySpaced"> 0 0 0 0.3 0 0 0.6 0 0 1 0 0 </E>'
                                 "</CURVED></GEOMETRY>"))
    with pytest.raises(SessionError):  # a curved face
        read_session(txt.replace("</GEOMETRY>", '<CURVED><F ID="0" FACEID="0" NUMPOINTS="3" '
                                 'TYPE="PolyEvenlySpaced"> 0 0 0 </F></CURVED></GEOMETRY>'))
    s = read_session(txt.replace('<D VAR="u"', '<R VAR="u"'))  # Robin without PRIMCOEFF
    with pytest.raises(SessionError):
        SessionMesh(s)
    # an unknown boundary condition kind
    from nektar_b200.session import with_conditions
    with pytest.raises(SessionError):
        SessionMesh(read_session(with_conditions(
            write_box_session("tet", 1, 4, 1.0, U, F, U),
            [([1, 2, 3, 4, 5], "D", U, None), ([6], "P", "0", None)])))


def test_fld_round_trip(tmp_path):
    from nektar_b200.fieldio import read_fld, write_fld
    s = _session(2, 5, seed=2)
    m = SessionMesh(s)
    coeffs = np.random.default_rng(1).uniform(-1, 1, m.nelmt * m.nc)
    out = str(tmp_path / "sol.fld")
    write_fld(out, m, {"u": coeffs})
    assert sorted(os.listdir(out)) == ["Info.xml", "P0000000.fld"]
    (d,) = read_fld(out)
    assert d["SHAPE"] == "Hexahedron" and d["NUMMODESPERDIR"] == "UNIORDER:5,5,5"
    assert d["COMPRESSED"] == "B64Z-LittleEndian" and d["BITSIZE"] == "64"
    assert d["ids"] == list(range(8)) and d["fields"] == ["u"]
    assert np.array_equal(d["data"], coeffs)


# --------------------------------------------------------------------------
# prisms and tetrahedra
# --------------------------------------------------------------------------
from nektar_b200.session import write_box_session  # noqa: E402

UQ = "x*x + 2*y*z - z"  # in every P >= 2 space: the discrete solution is exact
FQ = "2 - Lambda*(x*x + 2*y*z - z)"  # laplacian(u) - lambda u
REF_PRISM = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Prism.xml")
REF_TET = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Tet.xml")
REF_PRISM_VARP = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Prism_VarP.xml")
REF_TET_VARP = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Tet_VarP.xml")
REF_ALLBCS = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Hex_AllBCs_P6.xml")
REF_PRISM_DEF = ref_path("library/Demos/MultiRegions/Tests/Helmholtz3D_Prism_Deformed.xml")


@pytest.mark.parametrize("shape", ["prism", "tet"])
def test_collapsed_geometry_and_continuity(shape):
    s = read_session(write_box_session(shape, 2, 6, 1.0, U, F, U, shuffle_seed=5))
    m = SessionMesh(s)
    c = m.collections[0]
    assert np.isclose(m.quad_weights().sum(), 1.0)
    To = dict(c.T)
    To["w"] = c.T["ws"]
    for d in range(3):  # the chain rule through df and the collapsed factors
        g = O.physderiv(shape, c.nq, c.nelmt, To["D"], To["z"], c.df, c.xyz[d], True)
        for k, gk in enumerate(g):
            assert np.abs(gk - (1.0 if k == d else 0.0)).max() < 1e-12
    assert (m.sign < 0).any()
    xg = np.random.default_rng(3).uniform(-1, 1, m.nglob)
    u = O.bwdtrans(shape, c.nm, c.nq, c.nelmt, c.T["b"], m.sign * xg[m.gmap])
    vals = defaultdict(list)
    for p, v in zip(np.round(m.xyz.T, 9), u):
        vals[tuple(p)].append(v)
    assert max(max(v) - min(v) for v in vals.values()) < 1e-14


@pytest.mark.parametrize("shape,seed", [("hex", 7), ("prism", 2), ("tet", 4), ("hexprism", 1)])
def test_oracle_solve_reproduces_polynomial_solution(shape, seed):
    s = read_session(write_box_session(shape, 2, 4, 1.5, UQ, FQ, UQ, shuffle_seed=seed))
    _, linf, l2 = oracle_helm_solve(s)
    assert linf < 1e-12 and l2 < 1e-13


def test_incompatible_triangle_orientation_is_rejected():
    txt = write_box_session("tet", 1, 3, 1.0, U, F, U)
    s = read_session(txt)
    g = s.geometry
    # give one tetrahedron a rotated vertex order: its triangles now collapse
    # towards other vertices than their neighbours'
    shape, fs = g.elements[0]
    g.elements[0] = (shape, [fs[3], fs[0], fs[1], fs[2]])
    with pytest.raises(SessionError):
        SessionMesh(s)


@pytest.mark.skipif(not os.path.exists(REF_PRISM), reason="reference tree not mounted")
@pytest.mark.parametrize("path,record,tol", [
    # Helmholtz3D_CG_Prism.tst: L2, Linf, tolerance 1e-9
    (REF_PRISM, (0.000385246, 0.00539787), (1e-9, 1e-9)),
    # Helmholtz3D_CG_Tet.tst: L2 (tolerance 1e-8), Linf (1e-9)
    (REF_TET, (8.458e-05, 0.000862348), (1e-8, 1e-9)),
    # Helmholtz3D_CG_Prism_VarP.tst (orders 4, 5, 6 by composite): tolerance 1e-9
    (REF_PRISM_VARP, (0.000292496, 0.00539787), (1e-9, 1e-9)),
    # Helmholtz3D_CG_Tet_VarP.tst (orders 3, 4, 5, 6): L2 (tolerance 1e-7), Linf (1e-6)
    (REF_TET_VARP, (0.00416454, 0.0313733), (1e-7, 1e-6)),
    # Helmholtz3D_CG_Hex_AllBCs.tst (Dirichlet, Neumann and Robin sides): tolerance 1e-12
    (REF_ALLBCS, (0.000416575, 0.000871589), (1e-12, 1e-12)),
    # Helmholtz3D_CG_Prism_Deformed.tst (two quadratic curved edges): tolerance 1e-9
    (REF_PRISM_DEF, (8.88011e-06, 7.59576e-05), (1e-9, 1e-9)),
])
def test_reference_prism_tet_sessions_reproduce_their_records(path, record, tol):
    """The reference's own Prism / Tet regression sessions reproduce their
    recorded errors, including the reference's Dirichlet procedure on
    triangular faces (Radau -> GLL edge interpolation, boundary expansions
    grouped by type, face by face overwrites, copies to elements that only
    touch the boundary), in the VarP sessions variable order (edges and faces
    with the modes of their lowest-order element, the others of sign 0,
    Dirichlet faces projected at their element's order), and in AllBCs the
    Neumann and Robin terms (boundary inner products in the forcing,
    PRIMCOEFF-weighted face mass matrices in the operator), and in
    Prism_Deformed quadratic curved edges (the elements' maps with the edges'
    mode-2 coefficients, the boundary faces projected on their curved maps
    and grouped as deformed)."""
    _, linf, l2 = oracle_helm_solve(read_session(path))
    # the regression tester reads the demo's output, printed by cout with its
    # default six significant digits (Helmholtz3D.cpp: cout << vL2Error)
    printed = lambda v: float("%g" % v)  # noqa: E731
    assert abs(printed(l2) - record[0]) < tol[0] and abs(printed(linf) - record[1]) < tol[1]


def test_fld_mixed_mesh_has_one_block_per_collection(tmp_path):
    from nektar_b200.fieldio import read_fld, write_fld
    m = SessionMesh(read_session(write_box_session("hexprism", 2, 4, 1.0, U, F, U)))
    coeffs = np.arange(m.nloc, dtype=np.float64)
    write_fld(str(tmp_path / "m.fld"), m, {"u": coeffs})
    blocks = read_fld(str(tmp_path / "m.fld"))
    assert [b["SHAPE"] for b in blocks] == ["Hexahedron", "Prism"]
    assert blocks[1]["BASIS"] == "Modified_A,Modified_A,Modified_B"
    assert np.array_equal(np.concatenate([b["data"] for b in blocks]), coeffs)


def test_linear_solver_from_solver_info():
    from nektar_b200.helmsolve import linear_solver
    assert linear_solver({}) == ("full", "diagonal")
    assert linear_solver({"GlobalSysSoln": "IterativeStaticCond",
                          "Preconditioner": "LowEnergyBlock"}) == ("staticcond", "lowenergy")
    assert linear_solver({"GlobalSysSoln": "DirectStaticCond"}) == ("staticcond", "diagonal")
    # the reference's *_iter_ml.tst settings: multi-level condensation of the
    # same system, with the one-level records
    for k in ("Iterative", "Direct", "Xxt", "PETSc"):
        assert linear_solver({"GlobalSysSoln": k + "MultiLevelStaticCond"}) == \
            ("staticcond", "diagonal")
    with pytest.raises(ValueError):
        linear_solver({"GlobalSysSoln": "IterativeFull", "Preconditioner": "Block"})
    with pytest.raises(ValueError):
        linear_solver({"Preconditioner": "FullLinearSpace"})


def test_fld_variable_order_blocks(tmp_path):
    """One ELEMENTS block per collection, each with its own order."""
    from nektar_b200.fieldio import read_fld, write_fld
    from nektar_b200.session import with_orders
    m = SessionMesh(read_session(with_orders(write_box_session("tet", 2, 4, 1.0, U, F, U),
                                             [3, 5], seed=2)))
    coeffs = np.arange(m.nloc, dtype=np.float64)
    write_fld(str(tmp_path / "v.fld"), m, {"u": coeffs})
    blocks = read_fld(str(tmp_path / "v.fld"))
    assert [b["NUMMODESPERDIR"] for b in blocks] == ["UNIORDER:3,3,3", "UNIORDER:5,5,5"]
    assert sorted(i for b in blocks for i in b["ids"]) == list(range(48))
    assert np.array_equal(np.concatenate([b["data"] for b in blocks]), coeffs)


def test_weak_terms_do_not_depend_on_element_frames():
    """Neumann and Robin faces in rotated element frames (signs in the map):
    the same discrete solution, so the same errors."""
    from nektar_b200.session import ALL_BCS, with_conditions
    errs = []
    for seed in (None, 4, 7):
        s = read_session(with_conditions(write_hex_box_session(2, 5, 1.0, U, F, U,
                                                               shuffle_seed=seed), ALL_BCS))
        _, linf, l2 = oracle_helm_solve(s)
        errs.append((l2, linf))
    for l2, linf in errs[1:]:
        assert abs(l2 - errs[0][0]) < 1e-10 * errs[0][0] and abs(linf - errs[0][1]) < 1e-10


def test_robin_blocks_are_face_mass_matrices():
    """A Robin face's block is PRIMCOEFF times the face mass matrix of the
    global functions on it: symmetric, positive definite, and the sum of the
    vertex functions (the constant 1 on the face) integrates to the area."""
    from nektar_b200.session import ALL_BCS, with_conditions
    s = read_session(with_conditions(write_hex_box_session(2, 5, 1.0, U, F, U, shuffle_seed=4),
                                     ALL_BCS))
    m = SessionMesh(s)
    _, robin = m.weak_terms()
    assert robin
    for dofs, M, loc in robin:
        assert np.abs(M - M.T).max() < 1e-15 and np.linalg.eigvalsh(M)[0] > 0
        one = np.zeros(dofs.size)
        one[:4] = 1.0  # the four vertex functions come first
        prim = 2.0 if M.sum() > 0 and abs(one @ M @ one - 2 * 0.25) < 1e-12 else 3.0
        assert abs(one @ M @ one - prim * 0.25) < 1e-12  # faces of a 2^3 box: area 1/4


def _curve_session(shape="hex", n=2, nm=5, seed=3, bulge=(0.0, 0.0, 0.08)):
    """A box session with quadratic curves on the edges of the z = 1 face
    along x and on one interior edge."""
    s = read_session(write_box_session(shape, n, nm, 1.0, U, F, U, shuffle_seed=seed))
    g = s.geometry
    P = lambda v: np.asarray(g.vertices[v], dtype=np.float64)  # noqa: E731
    for e, (a, b) in g.edges.items():
        pa, pb = P(a), P(b)
        top = pa[2] == 1.0 and pb[2] == 1.0 and pa[1] == pb[1] and pa[0] != pb[0]
        inner = np.allclose(pa, [0.5, 0.5, 0.5]) and pb[2] == 0.5 and pb[1] == 0.5
        if top or inner:
            mid = 0.5 * (pa + pb) + np.asarray(bulge) * (1 if top else -0.5)
            g.curved_edges[e] = np.array([pa, mid, pb])
    return s


@pytest.mark.parametrize("shape", ["hex", "prism"])
def test_curved_edges_in_the_element_maps(shape):
    """Elements holding a curved edge take the quadratic through its three
    points: quadrature points on the edge lie on the curve, the map stays
    invertible, and the volume changes by the bulge's swept volume."""
    s = _curve_session(shape)
    assert s.geometry.curved_edges
    m = SessionMesh(s)
    straight = SessionMesh(read_session(write_box_session(shape, 2, 5, 1.0, U, F, U,
                                                          shuffle_seed=3)))
    vol, vol0 = m.quad_weights().sum(), straight.quad_weights().sum()
    assert all(c.jac.min() > 0 for c in m.collections)
    # the top face bulges outwards by 0.08 (1 - s^2) across every element
    # (s its local x coordinate): 0.08 * 2/3 of volume; the interior curve
    # moves as much volume into one element as out of its neighbour
    assert abs(vol - vol0 - 0.08 * 2.0 / 3.0) < 1e-12
    for c in m.collections:  # points on a curved edge lie on its quadratic
        if c.curves and any(c.curves):
            assert c.deformed


@pytest.mark.parametrize("shape", ["prism", "tet", "hexprism"])
def test_weak_terms_on_triangles_converge(shape):
    """Neumann and Robin data on triangular faces (the prism and tet boxes'
    y = 0 / y = 1 sides): frame-independent errors that fall spectrally with
    the order, as a consistent discretisation's must."""
    from nektar_b200.session import ALL_BCS, with_conditions
    errs = {}
    for nm in (4, 6, 8):
        for seed in (None, 5):
            s = read_session(with_conditions(write_box_session(shape, 2, nm, 1.0, U, F, U,
                                                               shuffle_seed=seed), ALL_BCS))
            m = SessionMesh(s)
            assert any(g_kind == "T" for g_kind in (s.geometry.faces[f][0] for f in m._face_weak))
            errs[(nm, seed)] = oracle_helm_solve(s, m)[2]
        assert abs(errs[(nm, None)] - errs[(nm, 5)]) < 1e-9 * errs[(nm, None)]
    assert errs[(6, None)] < 1e-2 * errs[(4, None)] and errs[(8, None)] < 1e-2 * errs[(6, None)]


def _explicit_expansions(txt, override=None):
    """The session text with every TYPE="MODIFIED" expansion written out as
    the bases and points it stands for (override: attributes to replace)."""
    import xml.etree.ElementTree as ET
    root = ET.fromstring(txt)
    comps = {int(c.get("ID")): c.text.strip()[0] for c in root.find("GEOMETRY").find("COMPOSITE")}
    std = {"H": ("Modified_A,Modified_A,Modified_A",
                 "GaussLobattoLegendre,GaussLobattoLegendre,GaussLobattoLegendre", (1, 1, 1)),
           "R": ("Modified_A,Modified_A,Modified_B",
                 "GaussLobattoLegendre,GaussLobattoLegendre,GaussRadauMAlpha1Beta0", (1, 1, 0)),
           "A": ("Modified_A,Modified_B,Modified_C",
                 "GaussLobattoLegendre,GaussRadauMAlpha1Beta0,GaussRadauMAlpha2Beta0", (1, 0, 0))}
    for e in root.find("EXPANSIONS").findall("E"):
        nm = int(e.get("NUMMODES"))
        letter = comps[int(e.get("COMPOSITE").strip()[2:-1].split(",")[0].split("-")[0])]
        b, p, extra = std[letter]
        del e.attrib["TYPE"]
        e.set("BASISTYPE", b)
        e.set("POINTSTYPE", p)
        e.set("NUMMODES", ",".join([str(nm)] * 3))
        e.set("NUMPOINTS", ",".join(str(nm + x) for x in extra))
        for k, v in (override or {}).items():
            e.set(k, v)
    return ET.tostring(root, encoding="unicode")


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_explicit_expansions_read_as_their_type(shape):
    """An expansion written out as bases and points (BASISTYPE, NUMMODES,
    POINTSTYPE, NUMPOINTS) that is the standard modified expansion reads as
    TYPE="MODIFIED" does: the same mesh and the same solution; per-direction
    orders (the reference's Hex_Heterogeneous session) and other point sets
    are refused by name."""
    txt = write_box_session(shape, 2, 4, 1.0, U, F, U, shuffle_seed=2)
    s0, s1 = read_session(txt), read_session(_explicit_expansions(txt))
    m0, m1 = SessionMesh(s0), SessionMesh(s1)
    assert [(c.shape, c.nm, c.nq) for c in m0.collections] == \
        [(c.shape, c.nm, c.nq) for c in m1.collections]
    assert np.array_equal(m0.gmap, m1.gmap) and np.array_equal(m0.sign, m1.sign)
    x0, _, _ = oracle_helm_solve(s0)
    x1, _, _ = oracle_helm_solve(s1)
    assert np.array_equal(x0, x1)
    with pytest.raises(SessionError, match="per-direction orders"):
        read_session(_explicit_expansions(txt, {"NUMMODES": "4,5,6"}))
    with pytest.raises(SessionError, match="not the standard modified expansion"):
        read_session(_explicit_expansions(txt, {"NUMPOINTS": "7,7,7"}))


def _bulged_top(txt, amp, with_faces=True, z0=1.0):
    """The box session with its plane z = z0 moved to
    z = z0 + amp x (1 - x) y (1 - y): the plane's vertices moved, its edges
    given their quadratic curves and (with_faces) its quadrilaterals their
    3 x 3 points in the CURVED section (MeshGraphIOXml's E and F records)."""
    import xml.etree.ElementTree as ET
    g = read_session(txt).geometry
    bump = lambda x, y: z0 + amp * x * (1 - x) * y * (1 - y)  # noqa: E731
    top = {v for v, p in g.vertices.items() if abs(p[2] - z0) < 1e-12}
    P = {v: np.array([p[0], p[1], bump(p[0], p[1]) if v in top else p[2]])
         for v, p in g.vertices.items()}
    root = ET.fromstring(txt)
    geo = root.find("GEOMETRY")
    for v in geo.find("VERTEX"):
        vid = int(v.get("ID"))
        v.text = "%.17g %.17g %.17g" % tuple(P[vid])
    cur = geo.find("CURVED")
    if cur is None:
        cur = ET.SubElement(geo, "CURVED")

    def on_top(x, y):
        return np.array([x, y, bump(x, y)])
    k = len(cur)
    for e, (a, b) in sorted(g.edges.items()):
        if a in top and b in top:
            m = 0.5 * (P[a] + P[b])
            pts = [P[a], on_top(m[0], m[1]), P[b]]
            c = ET.SubElement(cur, "E", ID=str(k), EDGEID=str(e), NUMPOINTS="3",
                              TYPE="PolyEvenlySpaced")
            c.text = " ".join("%.17g" % x for p in pts for x in p)
            k += 1
    if with_faces:
        for f, (kind, es) in sorted(g.faces.items()):
            vs = {v for e in es for v in g.edges[e]}
            if kind != "Q" or not vs <= top:
                continue
            # the face's vertex cycle v0 v1 v2 v3 and its points in tensor order
            cyc = [g.edges[es[0]][0], g.edges[es[0]][1]]
            while len(cyc) < 4:
                cyc.append(next(w for e in es for w in g.edges[e]
                                if cyc[-1] in g.edges[e] and w not in cyc))
            v0, v1, v3 = P[cyc[0]], P[cyc[1]], P[cyc[3]]
            pts = []
            for t in (0.0, 0.5, 1.0):
                for sv in (0.0, 0.5, 1.0):
                    xy = v0[:2] + sv * (v1[:2] - v0[:2]) + t * (v3[:2] - v0[:2])
                    pts.append(on_top(*xy))
            c = ET.SubElement(cur, "F", ID=str(k), FACEID=str(f), NUMPOINTS="9",
                              TYPE="PolyEvenlySpaced")
            c.text = " ".join("%.17g" % x for p in pts for x in p)
            k += 1
    return ET.tostring(root, encoding="unicode")


@pytest.mark.parametrize("shape", ["hex", "prism"])
def test_curved_faces_bend_the_element_maps(shape):
    """Quadratic curved faces (CURVED F records of 3 x 3 points): the (2, 2)
    mode of each curved quadrilateral joins the element maps of both its
    elements and the boundary-face maps, so a top surface bulged by a
    biquadratic is reproduced exactly (the domain's volume 1 + amp/36; a
    linear solution, Dirichlet data projected on the curved faces, solved
    to rounding), where curved edges alone miss the bulge."""
    amp = 0.8
    ul, fl = "x + 2*y + 3*z", "-Lambda*(x + 2*y + 3*z)"
    base = write_box_session(shape, 2, 4, 1.0, ul, fl, ul, shuffle_seed=1)
    s = read_session(_bulged_top(base, amp))
    assert s.geometry.curved_faces
    m = SessionMesh(s)
    assert abs(m.quad_weights().sum() - (1.0 + amp / 36.0)) < 1e-13
    _, linf, l2 = oracle_helm_solve(s, m)
    assert linf < 1e-11 and l2 < 1e-12, (linf, l2)
    me = SessionMesh(read_session(_bulged_top(base, amp, with_faces=False)))
    assert abs(me.quad_weights().sum() - (1.0 + amp / 36.0)) > 1e-4
    # a curved interior plane: both elements of every curved face take its
    # mode, so the maps still meet (the volume stays 1, the linear solution
    # stays exact)
    si = read_session(_bulged_top(base, 0.6 * amp, z0=0.5))
    mi = SessionMesh(si)
    assert abs(mi.quad_weights().sum() - 1.0) < 1e-13
    _, linf, l2 = oracle_helm_solve(si, mi)
    assert linf < 1e-11 and l2 < 1e-12, (linf, l2)


def test_curved_face_records_are_checked():
    """A curved face must have its vertices as corners; curves beyond
    quadratic order are refused by name."""
    base = write_box_session("hex", 1, 3, 1.0, U, F, U)
    txt = _bulged_top(base, 0.5)
    bad = txt.replace('NUMPOINTS="9"', 'NUMPOINTS="16"', 1)
    with pytest.raises(SessionError, match="quadratic curves only"):
        read_session(bad)
    import re
    m = re.search(r'(<F ID="\d+" FACEID="\d+" NUMPOINTS="9" TYPE="PolyEvenlySpaced">)([^<]*)', txt)
    vals = m.group(2).split()
    vals[0] = str(float(vals[0]) + 0.25)
    moved = txt.replace(m.group(0), m.group(1) + " ".join(vals))
    with pytest.raises(SessionError, match="vertices as corners"):
        read_session(moved)


@pytest.mark.parametrize("shape", ["hex", "prism"])
def test_face_bubbles_are_the_faces_own_modes(shape):
    """Each quadrilateral face's bubble (meshgraph.face_bubble) is
    (1 - s^2)(1 - t^2)/16 on its own face, zero on every other face, and its
    gradient is the derivative of the function."""
    from nektar_b200.meshgraph import STD_VERTS, face_bubble, topology
    V = STD_VERTS[shape]
    _, _, faces = topology(shape, 3)
    rng = np.random.default_rng(9)
    st = rng.uniform(-1, 1, (40, 2))
    for lf, (kind, frame, _) in enumerate(faces):
        if kind != "Q":
            continue
        o, a, c = (np.asarray(V[v], dtype=np.float64) for v in frame)
        # points of the face: o + (1+s)/2 (a - o) + (1+t)/2 (c - o)
        pts = o + np.outer(0.5 * (1 + st[:, 0]), a - o) + np.outer(0.5 * (1 + st[:, 1]), c - o)
        phi, _ = face_bubble(shape, lf, pts)
        want = 0.25 * (1 - st[:, 0] ** 2) * 0.25 * (1 - st[:, 1] ** 2)
        assert np.abs(phi - want).max() < 1e-14
        for lg, (kg, fg, _) in enumerate(faces):
            if lg == lf:
                continue
            og, ag, cg = (np.asarray(V[v], dtype=np.float64) for v in fg)
            if kg == "Q":
                q = og + np.outer(0.5 * (1 + st[:, 0]), ag - og) + \
                    np.outer(0.5 * (1 + st[:, 1]), cg - og)
            else:  # a triangle: barycentric points
                u = 0.5 * (1 + st)
                u = np.where((u.sum(axis=1) > 1)[:, None], 1 - u, u)
                q = og + np.outer(u[:, 0], ag - og) + np.outer(u[:, 1], cg - og)
            assert np.abs(face_bubble(shape, lf, q)[0]).max() < 1e-14
        x = rng.uniform(-0.9, 0.9, (30, 3))
        if shape == "prism":
            x[:, 2] = np.minimum(x[:, 2], -x[:, 0])  # inside: xi1 + xi3 <= 0
        _, g = face_bubble(shape, lf, x)
        h = 1e-6
        for d in range(3):
            e = np.zeros(3)
            e[d] = h
            fd = (face_bubble(shape, lf, x + e)[0] - face_bubble(shape, lf, x - e)[0]) / (2 * h)
            assert np.abs(fd - g[:, d]).max() < 1e-8
