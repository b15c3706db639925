"""FP64 setup of the product (nektar_b200/csrc/nkb_setup.cpp): quadrature,
modified bases, analytic geometric factors and the hex-box assembly map,
against the reference's Polylib (golden fixtures) and known answers."""
import os

import numpy as np
import pytest

import nektar_b200 as nb
from tests.helpers import GOLDEN, rel_l2

PB = dict(np.load(os.path.join(GOLDEN, "polylib_basis.npz")))


@pytest.mark.parametrize("ptype", [nb.GLL, nb.RADAU_A1, nb.RADAU_A2])
def test_points_match_reference_polylib(ptype):
    for n in range(2, 14):
        z, w, D = nb.points(ptype, n)
        assert np.abs(z - PB["z_%d_%d" % (ptype, n)]).max() < 1e-14
        assert rel_l2(w, PB["w_%d_%d" % (ptype, n)]) < 1e-13
        assert rel_l2(D, PB["D_%d_%d" % (ptype, n)]) < 1e-12


@pytest.mark.parametrize("ptype,alpha", [(nb.GLL, 0), (nb.RADAU_A1, 1), (nb.RADAU_A2, 2)])
def test_points_known_answers(ptype, alpha):
    """TestPolylib.cpp:244-290 style: exact integration against (1-z)^alpha
    and exact differentiation of polynomials."""
    from math import comb
    for n in range(3, 13):
        z, w, D = nb.points(ptype, n)
        deg = 2 * n - 3 if ptype == nb.GLL else 2 * n - 2
        for p in range(deg + 1):
            # int_{-1}^{1} (1-z)^alpha z^p dz, exactly, through the binomial series
            exact = sum(comb(alpha, a) * (-1) ** a *
                        ((1 - (-1) ** (p + a + 1)) / (p + a + 1)) for a in range(alpha + 1))
            assert abs(np.dot(w, z ** p) - exact) < 1e-12 * max(1.0, abs(exact))
        Dm = D.reshape(n, n).T  # Dm[i, k] = l_k'(z_i)
        for p in range(n):
            dp = p * z ** (p - 1) if p else np.zeros(n)
            assert np.abs(Dm @ z ** p - dp).max() < 1e-10 * max(1, p * p)


@pytest.mark.parametrize("btype,ptype", [(nb.MODIFIED_A, nb.GLL), (nb.MODIFIED_B, nb.RADAU_A1),
                                         (nb.MODIFIED_C, nb.RADAU_A2)])
def test_basis_matches_reference(btype, ptype):
    for nm in range(2, 12):
        n = nm + 1
        z, D = PB["z_%d_%d" % (ptype, n)], PB["D_%d_%d" % (ptype, n)]
        b, db = nb.basis(btype, nm, z, D)
        assert rel_l2(b, PB["b_%d_%d" % (btype, nm)]) < 1e-14
        assert rel_l2(db, PB["db_%d_%d" % (btype, nm)]) < 1e-13


def _curved(x, amp):
    s = np.sin(np.pi * x[0]) * np.sin(np.pi * x[1]) * np.sin(np.pi * x[2])
    return x + amp * s


@pytest.mark.parametrize("shape", ["hex", "prism", "tet"])
def test_geometry_volume_and_inverse(shape):
    m = nb.BoxMesh(shape, 2, 7, 9, amp=0.05, coords=True)
    W = np.einsum("i,j,k->kji", *m.T["ws"]).ravel()
    assert abs((m.jac.reshape(m.nelmt, -1) * W).sum() - 1.0) < 1e-5  # quadrature of a curved map
    assert m.jac.min() > 0
    # df rows are d xi_j/d x_k: check by differentiating x(xi) numerically through the
    # coordinates of the quadrature points, element by element, with the spectral D
    nq = m.nq
    Dm = [np.asarray(D).reshape(n, n).T for D, n in zip(m.T["D"], nq)]
    e = 1
    X = m.xyz[:, e * m.nt:(e + 1) * m.nt].reshape(3, nq[2], nq[1], nq[0])
    dX = [np.einsum("im,akjm->akji", Dm[0], X), np.einsum("jm,akmi->akji", Dm[1], X),
          np.einsum("km,amji->akji", Dm[2], X)]  # d x_a / d eta_d
    if shape == "hex":
        J = np.stack(dX, -1)  # [a, k, j, i, d]
        F = m.df[:, e * m.nt:(e + 1) * m.nt].reshape(3, 3, nq[2], nq[1], nq[0])  # [k, j, ...]
        prod = np.einsum("akjid,bdkji->abkji", J, F)  # sum_d dx_a/dxi_d dxi_d/dx_b
        err = np.abs(prod - np.eye(3)[:, :, None, None, None]).max()
        assert err < 1e-4  # spectral differentiation of the curved map with 9 points


def test_hex_box_assembly_sizes_and_multiplicity():
    m = nb.BoxMesh("hex", 32, 7, 8, amp=0.0, deformed=False)
    gmap, nglob, ndir = m.assembly()
    assert (nglob, ndir, len(gmap)) == (7189057, 221186, 11239424)  # sizes of the 32^3 P=6 box
    mult = np.bincount(gmap, minlength=nglob)
    assert set(np.unique(mult)) <= {1, 2, 4, 8}
    m2 = nb.BoxMesh("hex", 3, 4, 5)
    g2, ng2, nd2 = m2.assembly()
    # a global linear field gathered to the elements and evaluated is continuous:
    # vertex modes of neighbours at a shared corner share one global id
    e = g2.reshape(27, 4, 4, 4)  # [elem, r, q, p]
    # element 0's (p=1) face equals element 1's (p=0) face
    assert np.array_equal(e[0][:, :, 1], e[1][:, :, 0])
    assert np.array_equal(e[0][:, 1, :], e[3][:, 0, :])
    assert np.array_equal(e[0][1, :, :], e[9][0, :, :])
    # Dirichlet coefficients first: every boundary-face coefficient is < ndir
    assert e[0][:, :, 0].max() < nd2


def test_product_geometry_and_assembly_match_oracle_restatement():
    """The product's C++ setup against the oracle's numpy restatement."""
    from oracle import mesh as OM
    m = nb.BoxMesh("hex", 4, 5, 6, amp=0.05, coords=True)
    jac, df, xyz = OM.hex_box_geometry(4, m.T["z"][0], 0.05)
    assert rel_l2(m.jac, jac) < 1e-14
    assert rel_l2(m.df, df) < 1e-13
    assert rel_l2(m.xyz, xyz) < 1e-15
    g, ng, nd = m.assembly()
    go, ngo, ndo = OM.hex_box_assembly(4, 5)
    assert (ng, nd) == (ngo, ndo)
    assert np.array_equal(g, go)
