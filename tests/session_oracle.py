"""Test infrastructure: the Helmholtz solve of a session through the oracle
(oracle/nkoracle.c element operators, dense assembly with the session
mesh's signs, Dirichlet lifting, dense solve). It checks the host side of
the session path (reader, element frames, geometry, assembly, Dirichlet
projection) independently of the device, and against the reference's
recorded errors."""
import numpy as np

from oracle import oracle as O


def oracle_helm_solve(session, mesh=None):
    """(local coefficients, L_inf, L_2) of the session's Helmholtz solve."""
    from nektar_b200.meshgraph import SessionMesh
    m = mesh or SessionMesh(session)
    lam = session.parameters["Lambda"]
    To = dict(m.T)
    To["w"] = m.T["ws"]
    nc, ne = m.nc, m.nelmt
    K = np.zeros((ne, nc, nc))
    for j in range(nc):  # element matrices, one column per unit coefficient
        x = np.zeros(ne * nc)
        x[j::nc] = 1.0
        K[:, :, j] = O.helmholtz(m.shape, m.nm, m.nq, ne, To, m.jac, m.df, x, lam,
                                 True).reshape(ne, nc)
    G = np.zeros((m.nglob, m.nglob))
    gm, sg = m.gmap.reshape(ne, nc), m.sign.reshape(ne, nc)
    for e in range(ne):
        np.add.at(G, (gm[e][:, None], gm[e][None, :]), sg[e][:, None] * K[e] * sg[e][None, :])
    f = session.function("Forcing").evaluate(*m.xyz)
    b_loc = -O.iproduct(m.shape, m.nm, m.nq, ne, To["b"], To["w"], m.jac, f, True)
    b = np.zeros(m.nglob)
    np.add.at(b, m.gmap, m.sign * b_loc)
    xd = m.dirichlet_values()
    nd = m.ndir
    xg = np.concatenate([xd, np.linalg.solve(G[nd:, nd:], b[nd:] - G[nd:, :nd] @ xd)])
    xl = m.sign * xg[m.gmap]
    u = O.bwdtrans(m.shape, m.nm, m.nq, ne, To["b"], xl)
    ue = session.function("ExactSolution").evaluate(*m.xyz)
    W = m.quad_weights()
    return xl, float(np.max(np.abs(u - ue))), float(np.sqrt(np.sum(W * (u - ue) ** 2)))
