"""Test infrastructure only (the oracle): numpy restatement of the structured
curved hex box used by the benchmarks and tests, independent of the
product's C++ setup (nektar_b200/csrc/nkb_setup.cpp), so that

  * tests can check the product's geometric factors and assembly map, and
  * the reference arm of bench.py builds its inputs without product code.

Geometry as GeomFactors::ComputeJac / ComputeDerivFactors define it
(SpatialDomains/GeomFactors.cpp:248-477): jac = |det dx/dxi|,
df[k*3 + j] = d xi_j / d x_k, in the Collections layout of
CoalescedGeomData::GetJac / GetDerivFactors (9 rows of nelmt*nqtot), with the
analytic Jacobian of x' = x + amp sin(pi x) sin(pi y) sin(pi z).

Assembly: the C0 numbering of AssemblyMapCG (AssemblyMap/AssemblyMapCG.cpp
:1512-2045) specialised to an aligned box of Modified_A hexes, Dirichlet
(boundary) coefficients first.
"""
import numpy as np


def hex_box_geometry(n, z, amp, chunk=4096):
    """jac (nelmt*nt,), df (9, nelmt*nt) and coordinates (3, nelmt*nt) of the
    n^3 hex box at the 1-D points z (same in every direction)."""
    nq = len(z)
    nt = nq ** 3
    ne = n ** 3
    h = 1.0 / n
    jac = np.empty(ne * nt)
    df = np.empty((9, ne * nt))
    xyz = np.empty((3, ne * nt))
    zi = 0.5 * (np.asarray(z) + 1.0)
    # reference point (i, j, k) offsets within a cell, i fastest
    oi = np.tile(zi, nq * nq)
    oj = np.tile(np.repeat(zi, nq), nq)
    ok = np.repeat(zi, nq * nq)
    for e0 in range(0, ne, chunk):
        e = np.arange(e0, min(ne, e0 + chunk))
        cx, cy, cz = e % n, (e // n) % n, e // (n * n)
        x = ((cx[:, None] + oi[None, :]) * h).ravel()
        y = ((cy[:, None] + oj[None, :]) * h).ravel()
        zz = ((cz[:, None] + ok[None, :]) * h).ravel()
        sx, sy, sz = np.sin(np.pi * x), np.sin(np.pi * y), np.sin(np.pi * zz)
        cxp, cyp, czp = np.cos(np.pi * x), np.cos(np.pi * y), np.cos(np.pi * zz)
        S = sx * sy * sz
        dS = [np.pi * cxp * sy * sz, np.pi * sx * cyp * sz, np.pi * sx * sy * czp]
        # J[k][i] = d x'_k / d xi_i = h/2 (delta_ki + amp dS/dx_i)
        J = np.empty((3, 3, len(x)))
        for k in range(3):
            for i in range(3):
                J[k, i] = 0.5 * h * ((1.0 if k == i else 0.0) + amp * dS[i])
        det = (J[0, 0] * (J[1, 1] * J[2, 2] - J[1, 2] * J[2, 1]) -
               J[0, 1] * (J[1, 0] * J[2, 2] - J[1, 2] * J[2, 0]) +
               J[0, 2] * (J[1, 0] * J[2, 1] - J[1, 1] * J[2, 0]))
        Jt = np.moveaxis(J, 2, 0)  # (npts, 3, 3)
        inv = np.linalg.inv(Jt)    # inv[p, j, k] = d xi_j / d x_k
        sl = slice(e0 * nt, e0 * nt + len(x))
        jac[sl] = np.abs(det)
        for k in range(3):
            for j in range(3):
                df[k * 3 + j, sl] = inv[:, j, k]
        xyz[0, sl] = x + amp * S
        xyz[1, sl] = y + amp * S
        xyz[2, sl] = zz + amp * S
    return jac, df, xyz


def hex_box_assembly(n, nm):
    """(map, nglob, ndir): local -> global map of the n^3 box with nm modes.

    Per direction the 1-D dofs are the n+1 vertices and the n*(nm-2) edge
    interior modes of Modified_A; vertex v has id v*(nm-1), mode m >= 2 of
    cell c id c*(nm-1) + m-1. A 3-D coefficient is the triple of its 1-D ids;
    those touching the boundary of the box are Dirichlet and numbered first.
    """
    N1 = n * (nm - 1) + 1
    ids = np.arange(N1 ** 3)
    a, b, c = ids % N1, (ids // N1) % N1, ids // (N1 * N1)
    bnd = (a == 0) | (a == N1 - 1) | (b == 0) | (b == N1 - 1) | (c == 0) | (c == N1 - 1)
    num = np.empty(N1 ** 3, dtype=np.int64)
    nb = int(bnd.sum())
    num[bnd] = np.arange(nb)
    num[~bnd] = nb + np.arange(N1 ** 3 - nb)

    def d1(cell, p):
        return np.where(p == 0, cell * (nm - 1), np.where(p == 1, (cell + 1) * (nm - 1),
                                                          cell * (nm - 1) + p - 1))

    e = np.arange(n ** 3)
    cx, cy, cz = e % n, (e // n) % n, e // (n * n)
    m = np.arange(nm ** 3)
    p, q, r = m % nm, (m // nm) % nm, m // (nm * nm)
    g = (d1(cx[:, None], p[None, :]) + N1 * (d1(cy[:, None], q[None, :]) +
                                           N1 * d1(cz[:, None], r[None, :])))
    return num[g].ravel().astype(np.int32), N1 ** 3, nb


def csr_from_map(gmap, nglob):
    """global -> local CSR (row pointers, local indices) for the assemble."""
    order = np.argsort(gmap, kind="stable")
    ptr = np.zeros(nglob + 1, dtype=np.int64)
    np.add.at(ptr, gmap.astype(np.int64) + 1, 1)
    return np.cumsum(ptr).astype(np.int32), order.astype(np.int64)
