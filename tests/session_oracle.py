"""Test infrastructure: the Helmholtz solve of a session through the oracle
(oracle/nkoracle.c element operators, dense assembly with the session
mesh's signs, Dirichlet lifting, dense solve). It checks the host side of
the session path (reader, element frames, geometry, assembly, Dirichlet
projection) independently of the device, and against the reference's
recorded errors."""
import numpy as np

from oracle import oracle as O


def oracle_system(session, m):
    """(element matrices per collection, local right-hand side, Robin
    blocks) of the session's Helmholtz problem from the oracle's element
    operators."""
    lam = session.parameters["Lambda"]
    f = session.function("Forcing").evaluate(*m.xyz)
    Ks, b_loc = [], []
    for c, fc in zip(m.collections, m.split(f, "phys")):
        To = dict(c.T)
        To["w"] = c.T["ws"]
        nc, ne = c.nc, c.nelmt
        K = np.zeros((ne, nc, nc))
        for j in range(nc):  # element matrices, one column per unit coefficient
            x = np.zeros(ne * nc)
            x[j::nc] = 1.0
            K[:, :, j] = O.helmholtz(c.shape, c.nm, c.nq, ne, To, c.jac, c.df, x, lam,
                                     True).reshape(ne, nc)
        Ks.append(K)
        b_loc.append(-O.iproduct(c.shape, c.nm, c.nq, ne, To["b"], To["w"], c.jac, fc, True))
    # Neumann / Robin: boundary inner products in the forcing, Robin face
    # mass matrices in the operator
    rhs_w, robin = m.weak_terms()
    return Ks, np.concatenate(b_loc) + rhs_w, robin


def oracle_errors(session, m, x_loc):
    """(L_inf, L_2) of local coefficients against the session's exact
    solution (the oracle's backward transform, the mesh's quadrature)."""
    us = [O.bwdtrans(c.shape, c.nm, c.nq, c.nelmt, c.T["b"], xc)
          for c, xc in zip(m.collections, m.split(x_loc))]
    u = np.concatenate(us)
    ue = session.function("ExactSolution").evaluate(*m.xyz)
    W = m.quad_weights()
    return float(np.max(np.abs(u - ue))), float(np.sqrt(np.sum(W * (u - ue) ** 2)))


def oracle_helm_solve(session, mesh=None):
    """(local coefficients, L_inf, L_2) of the session's Helmholtz solve."""
    from nektar_b200.meshgraph import SessionMesh
    m = mesh or SessionMesh(session)
    lam = session.parameters["Lambda"]
    Ks, b_loc, robin = oracle_system(session, m)
    G = np.zeros((m.nglob, m.nglob))
    for c, K, gmc, sgc in zip(m.collections, Ks, m.split(m.gmap), m.split(m.sign)):
        gm, sg = gmc.reshape(c.nelmt, c.nc), sgc.reshape(c.nelmt, c.nc)
        for e in range(c.nelmt):
            np.add.at(G, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * K[e] * sg[e][None, :])
    for dofs, M, _ in robin:
        G[np.ix_(dofs, dofs)] += M
    # lifting with the local Dirichlet values element by element, as
    # GlobalLinSysIterativeFull::v_Solve does (GlobalLinSysIterativeFull.cpp:114-164)
    xdl = m.dirichlet_local()
    r_loc = b_loc - _apply_blocks(m, lam, xdl)
    b = np.zeros(m.nglob)
    np.add.at(b, m.gmap, m.sign * r_loc)
    for dofs, M, loc in robin:
        b[dofs] -= M @ (m.sign[loc] * xdl[loc])
    nd = m.ndir
    xg = np.concatenate([np.zeros(nd), np.linalg.solve(G[nd:, nd:], b[nd:])])
    xl = xdl + m.sign * xg[m.gmap]
    return (xl,) + oracle_errors(session, m, xl)


def _apply_blocks(m, lam, x_loc):
    """Element Helmholtz operators of every collection on a local vector."""
    out = []
    for c, xc in zip(m.collections, m.split(x_loc)):
        To = dict(c.T)
        To["w"] = c.T["ws"]
        out.append(O.helmholtz(c.shape, c.nm, c.nq, c.nelmt, To, c.jac, c.df, xc, lam, True))
    return np.concatenate(out)
