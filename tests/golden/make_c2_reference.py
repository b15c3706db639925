"""Run the reference CPU path once on the full-size FP64 solve workload (32^3
curved hexes, P=6, Q=8, lambda=1, PCG + Jacobi to a relative residual of
1e-10, manufactured solution u = sin(pi x) sin(pi y) sin(pi z)) and record
its iteration count, final residual and discretisation error in
tests/golden/c2_reference_cg.json, and a digest of its solutions (relative
residual 1e-10, and 1e-14: the converged FP64 solution) in
tests/golden/c2_reference_solution.npz: the local coefficients (Collections
layout, element-major) at 10000 seeded positions and the norms of the whole
local vectors. With --workload hex24_p8 the same for 24^3 curved hexes at
P=8, Q=10 (files c3_reference_*).

Everything timed or counted here is the reference's own arithmetic: its
MatrixFreeOps kernels compiled in place (oracle/_ref), driven by the
restated NekLinSysIterCG / AssemblyMapCG loop of oracle/ref_common.cpp;
inputs come from the oracle's numpy geometry (oracle/mesh.py). The bench's
CPU baseline times a bounded number of these iterations and scales by the
recorded count.

    python tests/golden/make_c2_reference.py [--workload hex24_p8]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import mesh as OM  # noqa: E402
from oracle import ref  # noqa: E402


def build(n=32, nm=7, amp=0.05, lam=1.0, nthreads=None):
    nthreads = nthreads or os.cpu_count()
    T, nq = ref.tables("hex", nm, nm + 1)
    jac, df, xyz = OM.hex_box_geometry(n, T["z"][0], amp)
    ne, nc = n ** 3, nm ** 3
    op = ref.RefOp("hex", "helmholtz", nm, nq, ne, T, jac=jac, df=df, deformed=True,
                   nthreads=nthreads)
    op.set_factors(lam)
    ipo = ref.RefOp("hex", "iproduct", nm, nq, ne, T, jac=jac, deformed=True, nthreads=nthreads)
    u = np.sin(np.pi * xyz[0]) * np.sin(np.pi * xyz[1]) * np.sin(np.pi * xyz[2])
    b_loc = np.zeros(ne * nc)
    ipo.apply((3 * np.pi ** 2 + lam) * u, b_loc)
    gmap, nglob, ndir = OM.hex_box_assembly(n, nm)
    aptr, aidx = OM.csr_from_map(gmap, nglob)
    b_glob = np.bincount(gmap, weights=b_loc, minlength=nglob)
    return dict(T=T, nq=nq, op=op, gmap=gmap, nglob=nglob, ndir=ndir, aptr=aptr, aidx=aidx,
                b_glob=b_glob, u=u, nc=nc, ne=ne, nthreads=nthreads, jac=jac, df=df)


WORKLOADS = {"hex32_p6": (32, 7, "c2", "32^3 curved hex, P=6, Q=8"),
             "hex24_p8": (24, 9, "c3", "24^3 curved hex, P=8, Q=10")}
DIGEST_SEED, DIGEST_COUNT = 2024, 10000


def digest_positions(nloc):
    """The seeded local positions the solution digest samples."""
    rng = np.random.default_rng(DIGEST_SEED)
    return np.sort(rng.choice(nloc, size=DIGEST_COUNT, replace=False)).astype(np.int64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="hex32_p6")
    n, nm, tag, name = WORKLOADS[ap.parse_args().workload]
    t0 = time.time()
    P = build(n=n, nm=nm)
    t1 = time.time()
    dloc = ref.helmholtz_diag(P["op"], P["nc"])
    dinv = 1.0 / np.bincount(P["gmap"], weights=dloc, minlength=P["nglob"])[P["ndir"]:]
    t2 = time.time()
    x, its, err = ref.pcg_solve(P["nglob"], P["ndir"], P["gmap"], None, P["aptr"], P["aidx"],
                                P["op"], dinv, P["b_glob"], tol=1e-10, maxit=20000,
                                nthreads=P["nthreads"])
    t3 = time.time()
    xt, its_t, err_t = ref.pcg_solve(P["nglob"], P["ndir"], P["gmap"], None, P["aptr"],
                                     P["aidx"], P["op"], dinv, P["b_glob"], tol=1e-14,
                                     maxit=20000, nthreads=P["nthreads"])
    # discretisation error at the quadrature points: BwdTrans of the solution
    T, nq = P["T"], P["nq"]
    nt = nq[0] * nq[1] * nq[2]
    bw = ref.RefOp("hex", "bwdtrans", nm, nq, P["ne"], T, nthreads=P["nthreads"])
    uh = np.zeros(P["ne"] * nt)
    bw.apply(x[P["gmap"]], uh)
    rms = float(np.sqrt(np.mean((uh - P["u"]) ** 2)))
    xl, xtl = x[P["gmap"]], xt[P["gmap"]]
    pos = digest_positions(xl.size)
    rec = {"workload": name + ", lambda=1, PCG+Jacobi, tol 1e-10",
           "iterations": int(its), "rel_residual": err, "rms_error_vs_exact": rms,
           "tight": {"tol": 1e-14, "iterations": int(its_t), "rel_residual": err_t,
                     "rel_l2_of_tol_1e-10_solution": float(np.linalg.norm(xl - xtl) /
                                                          np.linalg.norm(xtl))},
           "cpu_threads": P["nthreads"], "simd": ref.best_isa(),
           "seconds": {"setup": t1 - t0, "diagonal": t2 - t1, "solve": t3 - t2},
           "seconds_per_iteration": (t3 - t2) / its}
    with open(os.path.join(HERE, "%s_reference_cg.json" % tag), "w") as f:
        json.dump(rec, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "%s_reference_solution.npz" % tag),
                        seed=DIGEST_SEED, positions=pos, x=xl[pos], x_tight=xtl[pos],
                        norm=np.linalg.norm(xl), norm_tight=np.linalg.norm(xtl))
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
