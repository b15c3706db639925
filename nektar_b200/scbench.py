"""Static condensation against the full matrix-free solve on one GPU:
curved box of hexahedra, prisms or tetrahedra, P, random right-hand side, zero Dirichlet data; the full
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
    ap.add_argument("--shape", default="hex", choices=["hex", "prism", "tet"])
    ap.add_argument("--setup", default="device", choices=["device", "host"],
                    help="condensation on the device (nkb_condense) or in host numpy")
    ap.add_argument("--no-full", action="store_true",
                    help="condensed solves only (no full CG; for profiling them)")
    a = ap.parse_args()
    import nektar_b200 as nb
    from nektar_b200.staticcond import StaticCondSys, element_matrices
    nm = a.p + 1
    if a.shape == "hex":
        m = nb.BoxMesh("hex", a.n, nm, nm + 1, amp=0.05)
        gmap, nglob, ndir = m.assembly()
        sign, colls, what = None, [m], "curved hex box"
    else:  # straight-sided box session (the box assembly covers hexes only)
        from nektar_b200.meshgraph import SessionMesh
        from nektar_b200.session import read_session, write_box_session
        m = SessionMesh(read_session(write_box_session(a.shape, a.n, nm, 1.0, "0", "0", "0")))
        gmap, nglob, ndir, sign = m.gmap, m.nglob, m.ndir, m.sign
        colls, what = m.collections, "%s box session" % a.shape
    ops = []
    for c in colls:
        op = nb.Operator("helmholtz", c)
        op.set_factors(1.0)
        ops.append(op)
    nloc = sum(o.in_size for o in ops)
    import torch
    torch.zeros(1, device="cuda")  # the process's CUDA start-up is not set-up time
    torch.cuda.synchronize()
    b = np.random.default_rng(0).uniform(-1, 1, nloc)
    xf = rf = None
    if not a.no_full:
        full = nb.GlobalLinSys(ops, gmap, nglob, ndir, sign=sign)
        full.solve(b, tol=a.tol)  # warm (graphs)
        t0 = time.perf_counter()
        xf, rf = full.solve(b, tol=a.tol)
        full_wall = time.perf_counter() - t0
    t0 = time.perf_counter()
    # host set-up: element matrices copied back once and shared by the
    # condensed systems; device set-up: each system builds its own on the device
    K = [element_matrices(o) for o in ops] if a.setup == "host" else None
    t_mats = time.perf_counter() - t0
    out = {
        "workload": "%d^3 %s, P=%d, CG to %g" % (a.n, what, a.p, a.tol),
        "nglob": nglob, "setup": a.setup, "element_matrices_s": t_mats,
    }
    if rf is not None:
        out["full"] = {"precon": "diagonal", "iterations": rf.iterations,
                       "device_ms": rf.device_ms,
                       "ms_per_iteration": rf.device_ms / max(rf.iterations, 1),
                       "solve_wall_s": full_wall}
    for pc in a.precon.split(","):
        sc = StaticCondSys(ops, gmap, nglob, ndir, sign=sign, matrices=K, precon=pc,
                           setup=a.setup)
        sc.solve(b, tol=a.tol)
        t0 = time.perf_counter()
        xs, rs = sc.solve(b, tol=a.tol)
        wall = time.perf_counter() - t0
        d = sc.dense[0]
        d(np.zeros(d.in_size))
        ms = d.last_kernel_ms()
        nbm = sc.parts[0]["bm"].size
        dense_bytes = sc.parts[0]["ne"] * (nbm * nbm + 2 * nbm) * 8
        out["static_condensation_" + pc] = {
            "iterations": rs.iterations, "device_ms": rs.device_ms,
            "ms_per_iteration": rs.device_ms / max(rs.iterations, 1),
            "blocks": sc.nblocks, "boundary_dofs": sc.nglob_b,
            "setup_s": sc.setup_s, "setup_breakdown_s": sc.setup_breakdown,
            "solve_wall_s": wall,
            "dense_kernel_ms": ms, "dense_kernel_GB_s": dense_bytes / ms / 1e6,
            "schur_bytes": dense_bytes,
            "rel_l2_difference": (None if xf is None else
                                  float(np.linalg.norm(xs - xf) / np.linalg.norm(xf)))}
        sc.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
