"""Static condensation against the full matrix-free solve on one GPU:
curved hex box, P, random right-hand side, zero Dirichlet data; the full
solve with Jacobi, the condensed one with each preconditioner asked for
(diagonal, block, lowenergy).

    python -m nektar_b200.scbench --n 16 --p 6 [--tol 1e-10] [--precon diagonal,lowenergy]

Prints one JSON line: for every solver the CG iterations and the device time
of the solve (CUDA events); for static condensation also the host set-up
(element matrices from the device operator, condensation, low-energy
transform, blocks), the wall time of a solve (right-hand side condensation,
CG and back substitution, host buffers in and out as for the full solve), and
the dense block kernel's bandwidth.
"""
import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--p", type=int, default=6)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--precon", default="diagonal,block,lowenergy")
    a = ap.parse_args()
    import nektar_b200 as nb
    from nektar_b200.staticcond import StaticCondSys, element_matrices
    nm = a.p + 1
    m = nb.BoxMesh("hex", a.n, nm, nm + 1, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    b = np.random.default_rng(0).uniform(-1, 1, m.nelmt * m.nc)
    full = nb.GlobalLinSys([op], gmap, nglob, ndir)
    full.solve(b, tol=a.tol)  # warm (graphs)
    t0 = time.perf_counter()
    xf, rf = full.solve(b, tol=a.tol)
    full_wall = time.perf_counter() - t0
    t0 = time.perf_counter()
    K = [element_matrices(op)]  # shared by the condensed systems
    t_mats = time.perf_counter() - t0
    out = {
        "workload": "%d^3 curved hex, P=%d, CG to %g" % (a.n, a.p, a.tol),
        "nglob": nglob, "element_matrices_s": t_mats,
        "full": {"precon": "diagonal", "iterations": rf.iterations, "device_ms": rf.device_ms,
                 "ms_per_iteration": rf.device_ms / max(rf.iterations, 1),
                 "solve_wall_s": full_wall},
    }
    for pc in a.precon.split(","):
        sc = StaticCondSys([op], gmap, nglob, ndir, matrices=K, precon=pc)
        sc.solve(b, tol=a.tol)
        t0 = time.perf_counter()
        xs, rs = sc.solve(b, tol=a.tol)
        wall = time.perf_counter() - t0
        d = sc.dense[0]
        d(np.zeros(d.in_size))
        ms = d.last_kernel_ms()
        nbm = sc.parts[0]["bm"].size
        dense_bytes = m.nelmt * (nbm * nbm + 2 * nbm) * 8
        out["static_condensation_" + pc] = {
            "iterations": rs.iterations, "device_ms": rs.device_ms,
            "ms_per_iteration": rs.device_ms / max(rs.iterations, 1),
            "blocks": sc.nblocks, "boundary_dofs": sc.nglob_b,
            "setup_s": sc.setup_s, "solve_wall_s": wall,
            "dense_kernel_ms": ms, "dense_kernel_GB_s": dense_bytes / ms / 1e6,
            "schur_bytes": dense_bytes,
            "rel_l2_difference": float(np.linalg.norm(xs - xf) / np.linalg.norm(xf))}
        sc.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
