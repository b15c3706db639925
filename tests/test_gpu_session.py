"""Session solves on the device (operators and CG through the C ABI) against
the reference's recorded errors for Helmholtz3D_CG_Hex.tst (L2 1.11818e-07,
Linf 5.66374e-07, tolerance 1e-12) and against the oracle's dense solve."""
import pytest

from nektar_b200.helmsolve import helm_solve
from nektar_b200.session import read_session, write_hex_box_session
from tests.helpers import rel_l2
from tests.session_oracle import oracle_helm_solve

pytestmark = pytest.mark.gpu

U = "sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
F = "-(Lambda + 3*PI*PI/4)*sin(PI/2*x)*sin(PI/2*y)*sin(PI/2*z)"
HEX_L2, HEX_LINF = 1.11818e-07, 5.66374e-07


@pytest.mark.parametrize("seed", [None, 4, 9])
def test_device_solve_reproduces_reference_record(seed):
    s = read_session(write_hex_box_session(2, 6, 1.0, U, F, U, shuffle_seed=seed))
    r = helm_solve(s, tol=1e-14, maxit=2000, raise_on_maxit=False)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert r.rel_residual < 1e-12
    assert rel_l2(r.coeffs, xo) < 1e-11
    assert abs(r.l2 - HEX_L2) < 1e-12 and abs(r.linf - HEX_LINF) < 1e-12


def test_device_solve_converges_under_refinement():
    """P=5 on 2^3 and 6^3 rotated-frame meshes: the L2 error falls like
    h^(P+1) (factor 3^6 = 729 in exact arithmetic)."""
    errs = []
    for n in (2, 6):
        s = read_session(write_hex_box_session(n, 6, 1.0, U, F, U, shuffle_seed=n))
        r = helm_solve(s, tol=1e-13, maxit=5000, raise_on_maxit=False)
        errs.append(r.l2)
    assert errs[0] / errs[1] > 300


from nektar_b200.session import write_box_session  # noqa: E402

UQ = "x*x + 2*y*z - z"
FQ = "2 - Lambda*(x*x + 2*y*z - z)"


@pytest.mark.parametrize("shape,seed", [("prism", 3), ("tet", 5), ("hexprism", 2)])
def test_device_solve_matches_oracle_on_collapsed_and_mixed_meshes(shape, seed):
    s = read_session(write_box_session(shape, 2, 6, 1.0, U, F, U, shuffle_seed=seed))
    r = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert r.rel_residual < 1e-12
    assert rel_l2(r.coeffs, xo) < 1e-11
    assert abs(r.l2 - l2_o) < 1e-12 * max(1.0, l2_o) + 1e-13


@pytest.mark.parametrize("shape", ["hex", "prism", "tet", "hexprism"])
def test_device_solve_reproduces_polynomial_solution(shape):
    """A quadratic solution lies in the discrete space: the device solve on a
    larger mesh with rotated frames returns it to the solver tolerance."""
    s = read_session(write_box_session(shape, 4, 5, 2.0, UQ, FQ, UQ, shuffle_seed=6))
    r = helm_solve(s, tol=1e-13, maxit=3000)
    assert r.linf < 1e-10 and r.l2 < 1e-11


@pytest.mark.parametrize("soln,precon", [("IterativeStaticCond", "Diagonal"),
                                         ("IterativeStaticCond", "Block"),
                                         ("IterativeStaticCond", "LowEnergyBlock"),
                                         ("IterativeMultiLevelStaticCond", "Diagonal")])
def test_static_condensation_solvers_reproduce_reference_record(soln, precon):
    """-I GlobalSysSoln=IterativeStaticCond (or IterativeMultiLevelStaticCond,
    the *_iter_ml.tst setting) -I Preconditioner=...: the condensed solves
    give the Hex record's errors as the full solve does."""
    s = read_session(write_hex_box_session(2, 6, 1.0, U, F, U, shuffle_seed=4))
    info = {"GlobalSysSoln": soln, "Preconditioner": precon}
    r = helm_solve(s, tol=1e-14, maxit=2000, raise_on_maxit=False, solver_info=info)
    assert (r.solver, r.precon) == ("staticcond", {"Diagonal": "diagonal", "Block": "block",
                                                   "LowEnergyBlock": "lowenergy"}[precon])
    assert abs(r.l2 - HEX_L2) < 1e-12 and abs(r.linf - HEX_LINF) < 1e-12


@pytest.mark.parametrize("shape", ["prism", "tet", "hexprism"])
def test_lowenergy_session_solve_matches_full_solve(shape):
    s = read_session(write_box_session(shape, 2, 6, 1.0, U, F, U, shuffle_seed=3))
    rf = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False)
    info = {"GlobalSysSoln": "IterativeStaticCond", "Preconditioner": "LowEnergyBlock"}
    rl = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False, solver_info=info)
    assert rel_l2(rl.coeffs, rf.coeffs) < 1e-10
    assert abs(rl.l2 - rf.l2) < 1e-9 * rf.l2
    assert rl.iterations * 3 < rf.iterations


@pytest.mark.parametrize("shape", ["hex", "prism", "tet", "hexprism"])
def test_variable_order_session_matches_oracle(shape):
    """Elements of orders 4, 5 and 6 in one mesh (as the reference's *_VarP
    sessions): edges and faces carry their lowest-order element's modes, the
    other local modes have sign 0 in the gather, the assemble and the Jacobi
    diagonal; the device solve (full and condensed) matches the oracle's."""
    from nektar_b200.session import with_orders
    s = read_session(with_orders(write_box_session(shape, 2, 5, 1.0, U, F, U, shuffle_seed=3),
                                 [4, 6, 5], seed=1))
    r = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert len(r.mesh.collections) >= 3 and (r.mesh.sign == 0).any()
    assert rel_l2(r.coeffs, xo) < 1e-10
    assert abs(r.l2 - l2_o) < 1e-9 * l2_o and abs(r.linf - linf_o) < 1e-9 * linf_o
    for precon in ("Diagonal", "Block", "LowEnergyBlock"):
        # Block and LowEnergy over the modes of nonzero sign; LowEnergy with the
        # transforms of the highest order cut down to each element's
        # (ExtractLocMat) and the modes a lower-order neighbour lacks masked
        # (CreateVariablePMask), as Helmholtz3D_CG_Tet_VarP_iterLE.tst runs it
        rc = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False,
                        solver_info={"GlobalSysSoln": "IterativeStaticCond",
                                     "Preconditioner": precon})
        assert rc.converged and rel_l2(rc.coeffs, xo) < 1e-10, precon
        if precon == "Diagonal":
            it_diag = rc.iterations
    assert rc.iterations < it_diag


@pytest.mark.parametrize("info", [None, {"GlobalSysSoln": "IterativeStaticCond"},
                                  {"GlobalSysSoln": "IterativeStaticCond",
                                   "Preconditioner": "LowEnergyBlock"}])
@pytest.mark.parametrize("orders,shape", [(None, "hex"), ([4, 6], "hex"), (None, "prism"),
                                          (None, "tet")])
def test_neumann_robin_session_matches_oracle(info, orders, shape):
    """Dirichlet, Neumann and Robin sides (the reference's AllBCs
    conditions) in rotated element frames: the Robin face mass matrices as
    extra dense operators of the device CG (full solve) or folded into the
    element matrices (condensed solves) give the oracle's solution."""
    from nektar_b200.session import ALL_BCS, with_conditions, with_orders
    txt = (write_hex_box_session(3, 5, 1.0, U, F, U, shuffle_seed=4) if shape == "hex" else
           write_box_session(shape, 2, 5, 1.0, U, F, U, shuffle_seed=4))
    if orders:
        txt = with_orders(txt, orders, seed=3)
    s = read_session(with_conditions(txt, ALL_BCS))
    r = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False, solver_info=info)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert rel_l2(r.coeffs, xo) < 1e-10
    assert abs(r.l2 - l2_o) < 1e-9 * l2_o and abs(r.linf - linf_o) < 1e-9 * linf_o


@pytest.mark.parametrize("shape", ["hex", "prism"])
def test_curved_session_matches_oracle(shape):
    """Quadratic curved edges (on the boundary and inside): the device solve
    on the curved element maps matches the oracle's."""
    from tests.test_session import _curve_session
    s = _curve_session(shape)
    r = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert rel_l2(r.coeffs, xo) < 1e-10
    assert abs(r.l2 - l2_o) < 1e-9 * l2_o


@pytest.mark.parametrize("shape", ["hex", "prism"])
def test_curved_face_session_matches_oracle(shape):
    """Quadratic curved faces (a bulged top surface and a bulged interior
    plane): the device solve on those element maps, full and condensed,
    matches the oracle's."""
    from nektar_b200.session import write_box_session
    from tests.test_session import _bulged_top
    base = write_box_session(shape, 2, 5, 1.0, U, F, U, shuffle_seed=2)
    s = read_session(_bulged_top(_bulged_top(base, 0.8), 0.5, z0=0.5))
    assert s.geometry.curved_faces
    r = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False)
    xo, linf_o, l2_o = oracle_helm_solve(s, r.mesh)
    assert rel_l2(r.coeffs, xo) < 1e-10
    assert abs(r.l2 - l2_o) < 1e-9 * l2_o
    rc = helm_solve(s, tol=1e-14, maxit=3000, raise_on_maxit=False,
                    solver_info={"GlobalSysSoln": "IterativeStaticCond"})
    assert rel_l2(rc.coeffs, xo) < 1e-10
