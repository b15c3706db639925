"""Static condensation against the full matrix-free solve on one GPU:
curved hex box, P, PCG + Jacobi, random right-hand side, zero Dirichlet data.

    python -m nektar_b200.scbench --n 16 --p 6 [--tol 1e-10]

Prints one JSON line: for both solvers the CG iterations and the device time
of the solve (CUDA events); for static condensation also the host set-up
(element matrices from the device operator, condensation), the host
condensation of the right-hand side and back substitution, and the dense
block kernel's bandwidth.
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
    a = ap.parse_args()
    import nektar_b200 as nb
    from nektar_b200.staticcond import StaticCondSys
    nm = a.p + 1
    m = nb.BoxMesh("hex", a.n, nm, nm + 1, amp=0.05)
    gmap, nglob, ndir = m.assembly()
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.0)
    b = np.random.default_rng(0).uniform(-1, 1, m.nelmt * m.nc)
    full = nb.GlobalLinSys([op], gmap, nglob, ndir)
    full.solve(b, tol=a.tol)  # warm (graphs)
    xf, rf = full.solve(b, tol=a.tol)
    sc = StaticCondSys([op], gmap, nglob, ndir)
    sc.solve(b, tol=a.tol)
    t0 = time.perf_counter()
    xs, rs = sc.solve(b, tol=a.tol)
    wall = time.perf_counter() - t0
    d = sc.dense[0]
    x = np.zeros(d.in_size)
    d(x)
    ms = d.last_kernel_ms()
    nbm = sc.parts[0]["bm"].size
    dense_bytes = m.nelmt * (nbm * nbm + 2 * nbm) * 8
    print(json.dumps({
        "workload": "%d^3 curved hex, P=%d, PCG+Jacobi to %g" % (a.n, a.p, a.tol),
        "nglob": nglob, "boundary_dofs": sc.nglob_b,
        "full": {"iterations": rf.iterations, "device_ms": rf.device_ms,
                 "ms_per_iteration": rf.device_ms / max(rf.iterations, 1)},
        "static_condensation": {
            "iterations": rs.iterations, "device_ms": rs.device_ms,
            "ms_per_iteration": rs.device_ms / max(rs.iterations, 1),
            "setup_s": sc.setup_s, "solve_wall_s": wall,
            "dense_kernel_ms": ms, "dense_kernel_GB_s": dense_bytes / ms / 1e6,
            "schur_bytes": dense_bytes},
        "rel_l2_difference": float(np.linalg.norm(xs - xf) / np.linalg.norm(xf)),
    }), flush=True)


if __name__ == "__main__":
    main()
