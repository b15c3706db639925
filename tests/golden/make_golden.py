"""Generate the golden fixtures of tests/golden/*.npz from the reference's own
MatrixFreeOps kernels and Polylib, compiled in place into oracle/_ref by
`make -C oracle ref` (this needs the reference source tree, so it runs where
the reference is mounted; the fixtures are committed and travel instead).

    python tests/golden/make_golden.py           # the fixtures that are missing
    python tests/golden/make_golden.py --force   # all of them

Every case stores its seeded inputs, the reference-generated 1-D tables and
the reference kernels' outputs. Inputs follow the pattern of the reference's
Collections unit tests (TestHexCollection.cpp:4334-4605 and the Tet/Prism
analogues): a few elements, coefficients i+1 or seeded uniform[-1,1] values,
lambda = 1.5, regular and deformed geometry.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402

SPEC = {
    "hex": [(ref.MOD_A, ref.GLL, 0)] * 3,
    "prism": [(ref.MOD_A, ref.GLL, 0), (ref.MOD_A, ref.GLL, 0), (ref.MOD_B, ref.RADAU_A1, -1)],
    "tet": [(ref.MOD_A, ref.GLL, 0), (ref.MOD_B, ref.RADAU_A1, -1), (ref.MOD_C, ref.RADAU_A2, -1)],
}


def ref_tables(shape, nm, nq0):
    T = {"b": [], "db": [], "w": [], "ws": [], "z": [], "D": [], "ptype": []}
    nq = []
    for bt, pt, dq in SPEC[shape]:
        n = nq0 + dq
        z, w, D = ref.points(pt, n)
        b, db = ref.basis(bt, nm, pt, n)
        for k, v in (("b", b), ("db", db), ("w", w), ("ws", w * ref.weight_factor(pt)),
                     ("z", z), ("D", D), ("ptype", pt)):
            T[k].append(v)
        nq.append(n)
    return T, tuple(nq)


def ncoeffs(shape, nm):
    return {"hex": nm ** 3, "prism": nm * nm * (nm + 1) // 2,
            "tet": nm * (nm + 1) * (nm + 2) // 6}[shape]


def make_case(shape, nm, nq0, deformed, seed, ne=3):
    rng = np.random.default_rng(seed)
    T, nq = ref_tables(shape, nm, nq0)
    nt = nq[0] * nq[1] * nq[2]
    nc = ncoeffs(shape, nm)
    ncol = ne * nt if deformed else ne
    jac = rng.uniform(0.5, 1.5, ncol)
    df = rng.uniform(-1.0, 1.0, (9, ncol))
    x = np.arange(1, ne * nc + 1, dtype=np.float64)
    x_rand = rng.uniform(-1.0, 1.0, ne * nc)
    f = rng.uniform(-1.0, 1.0, ne * nt)
    f3 = rng.uniform(-1.0, 1.0, 3 * ne * nt)  # a vector field for IProductWRTDerivBase
    vel = rng.uniform(-1.0, 1.0, 3 * ne * nt)  # advection velocity for LinearADR
    # the harness takes weights already scaled as MatrixFree SetUpZW scales them
    T = dict(T)
    T["w_raw"], T["w"] = T["w"], T["ws"]
    out = {}
    op = ref.RefOp(shape, "bwdtrans", nm, nq, ne, T)
    y = np.zeros(ne * nt)
    op.apply(x_rand, y)
    out["bwdtrans"] = y
    op = ref.RefOp(shape, "iproduct", nm, nq, ne, T, jac=jac, deformed=deformed)
    y = np.zeros(ne * nc)
    op.apply(f, y)
    out["iproduct"] = y
    op = ref.RefOp(shape, "physderiv", nm, nq, ne, T, df=df, deformed=deformed)
    d = [np.zeros(ne * nt) for _ in range(3)]
    op.apply(f, *d)
    out["physderiv"] = np.stack(d)
    op = ref.RefOp(shape, "iproduct_deriv", nm, nq, ne, T, jac=jac, df=df, deformed=deformed)
    y = np.zeros(ne * nc)
    op.apply(f3, y)
    out["iproduct_deriv"] = y
    op = ref.RefOp(shape, "linear_adr", nm, nq, ne, T, jac=jac, df=df, deformed=deformed)
    op.set_adr(1.5, vel)
    y = np.zeros(ne * nc)
    op.apply(x, y)
    out["linear_adr"] = y
    diff = np.array([1.3, 0.2, 0.9, 0.1, -0.3, 1.1])
    for mode, tag in ((0, "helmholtz"), (1, "helmholtz_constdiff"), (2, "helmholtz_vardiff")):
        op = ref.RefOp(shape, "helmholtz", nm, nq, ne, T, jac=jac, df=df, deformed=deformed)
        op.set_factors(1.5, const_diff=diff if mode == 1 else None,
                       var_diff=diff if mode == 2 else None)
        y = np.zeros(ne * nc)
        op.apply(x, y)
        out[tag] = y
    arrays = {"nq": np.array(nq), "nm": np.array(nm), "ne": np.array(ne),
              "deformed": np.array(int(deformed)), "jac": jac, "df": df, "x": x,
              "x_rand": x_rand, "f": f, "f3": f3, "vel": vel, "lam": np.array(1.5), "diff": diff,
              "ptype": np.array(T["ptype"])}
    for k, src in (("b", "b"), ("db", "db"), ("w", "w_raw"), ("ws", "ws"), ("z", "z"),
                   ("D", "D")):
        for dd in range(3):
            arrays["%s%d" % (k, dd)] = T[src][dd]
    for k, v in out.items():
        arrays["out_" + k] = v
    return arrays


CASES = [(s, nm, nm + 1, dfm) for s in ("hex", "prism", "tet") for nm in (2, 3, 5)
         for dfm in (False, True)]
# the benchmark orders: Hex P=6 (nm 7, Q=8) and P=8 (nm 9, Q=10), Prism and Tet at
# nm 7; two elements each, to keep the fixtures small
CASES += [(s, nm, nm + 1, dfm) for s, nm in (("hex", 7), ("hex", 9), ("prism", 7), ("tet", 7))
          for dfm in (False, True)]
# over-integration as the reference's *_OverInt Collections tests set it up
# (TestHexCollection.cpp:4423-4470: 4 modes, 8 quadrature points per direction)
CASES += [(s, 4, 8, dfm) for s in ("hex", "prism", "tet") for dfm in (False, True)]


def main(force=False):
    """Writes the fixtures that are missing (all with force=True)."""
    for shape, nm, nq0, deformed in CASES:
        name = "%s_nm%d_nq%d_%s.npz" % (shape, nm, nq0, "deformed" if deformed else "regular")
        path = os.path.join(HERE, name)
        if os.path.exists(path) and not force:
            continue
        arrays = make_case(shape, nm, nq0, deformed, seed=1000 * nm + nq0 + int(deformed),
                           ne=3 if nm <= 5 else 2)
        np.savez_compressed(path, **arrays)
        print("wrote", name)
    if os.path.exists(os.path.join(HERE, "polylib_basis.npz")) and not force:
        return
    # quadrature / basis known answers from the reference Polylib
    pts = {}
    for pt in (ref.GLL, ref.RADAU_A1, ref.RADAU_A2):
        for n in range(2, 14):
            z, w, D = ref.points(pt, n)
            pts["z_%d_%d" % (pt, n)] = z
            pts["w_%d_%d" % (pt, n)] = w
            pts["D_%d_%d" % (pt, n)] = D
    for bt, pt in ((ref.MOD_A, ref.GLL), (ref.MOD_B, ref.RADAU_A1), (ref.MOD_C, ref.RADAU_A2)):
        for nm in range(2, 12):
            n = nm + 1
            b, db = ref.basis(bt, nm, pt, n)
            pts["b_%d_%d" % (bt, nm)] = b
            pts["db_%d_%d" % (bt, nm)] = db
    np.savez_compressed(os.path.join(HERE, "polylib_basis.npz"), **pts)
    print("wrote polylib_basis.npz")


if __name__ == "__main__":
    main(force="--force" in sys.argv[1:])
