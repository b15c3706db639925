"""Test infrastructure only (the oracle): ctypes wrapper over the plain-C
restatement oracle/nkoracle.c (built to oracle/_build/liboracle.so by
`make -C oracle`), plus small numpy helpers shared by the tests.

The checker, never the thing measured or shipped: only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
SHAPES = {"tet": 5, "prism": 7, "hex": 8}

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.or_ncoeffs.restype = ctypes.c_int
        L.or_bwdtrans.restype = None
        L.or_iproduct.restype = None
        L.or_physderiv.restype = None
        L.or_iproduct_deriv.restype = None
        L.or_linear_adr.restype = None
        L.or_helmholtz.restype = None
        L.or_pcg.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _arr3(tabs):
    tabs = [np.ascontiguousarray(t, dtype=np.float64) for t in tabs]
    return tabs, (_dp * 3)(*[_p(t) for t in tabs])


def ncoeffs(shape, nm):
    return lib().or_ncoeffs(SHAPES[shape], nm)


def bwdtrans(shape, nm, nq, nelmt, B, x):
    keep, Bp = _arr3(B)
    out = np.zeros(nelmt * nq[0] * nq[1] * nq[2])
    lib().or_bwdtrans(SHAPES[shape], nm, (ctypes.c_int * 3)(*nq), nelmt, Bp,
                      _p(np.ascontiguousarray(x)), _p(out))
    return out


def iproduct(shape, nm, nq, nelmt, B, w, jac, f, deformed):
    kb, Bp = _arr3(B)
    kw, Wp = _arr3(w)
    out = np.zeros(nelmt * ncoeffs(shape, nm))
    lib().or_iproduct(SHAPES[shape], int(deformed), nm, (ctypes.c_int * 3)(*nq), nelmt, Bp, Wp,
                      _p(np.ascontiguousarray(jac)), _p(np.ascontiguousarray(f)), _p(out))
    return out


def physderiv(shape, nq, nelmt, D, Z, df, f, deformed):
    kd, Dp = _arr3(D)
    kz, Zp = _arr3(Z)
    n = nelmt * nq[0] * nq[1] * nq[2]
    o0, o1, o2 = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().or_physderiv(SHAPES[shape], int(deformed), (ctypes.c_int * 3)(*nq), nelmt, Dp, Zp,
                       _p(np.ascontiguousarray(df)), _p(np.ascontiguousarray(f)), _p(o0), _p(o1),
                       _p(o2))
    return o0, o1, o2


def linear_adr(shape, nm, nq, nelmt, T, jac, df, lam, vel, x, deformed):
    """vel: the three velocity fields consecutively (3 * nelmt * nt values),
    lam the Collections-level lambda (the operator applies -lam)."""
    kb, Bp = _arr3(T["b"])
    kdb, dBp = _arr3(T["db"])
    kw, Wp = _arr3(T["w"])
    kd, Dp = _arr3(T["D"])
    kz, Zp = _arr3(T["z"])
    out = np.zeros(nelmt * ncoeffs(shape, nm))
    lib().or_linear_adr(SHAPES[shape], int(deformed), nm, (ctypes.c_int * 3)(*nq), nelmt, Bp, dBp,
                        Wp, Dp, Zp, _p(np.ascontiguousarray(jac)), _p(np.ascontiguousarray(df)),
                        ctypes.c_double(lam), _p(np.ascontiguousarray(vel)),
                        _p(np.ascontiguousarray(x)), _p(out))
    return out


def iproduct_deriv(shape, nm, nq, nelmt, T, jac, df, f, deformed):
    """f: the three physical fields consecutively (3 * nelmt * nt values)."""
    kb, Bp = _arr3(T["b"])
    kdb, dBp = _arr3(T["db"])
    kw, Wp = _arr3(T["w"])
    kz, Zp = _arr3(T["z"])
    out = np.zeros(nelmt * ncoeffs(shape, nm))
    lib().or_iproduct_deriv(SHAPES[shape], int(deformed), nm, (ctypes.c_int * 3)(*nq), nelmt,
                            Bp, dBp, Wp, Zp, _p(np.ascontiguousarray(jac)),
                            _p(np.ascontiguousarray(df)), _p(np.ascontiguousarray(f)), _p(out))
    return out


def helmholtz(shape, nm, nq, nelmt, T, jac, df, x, lam=1.0, deformed=True, diff_mode=0,
              diff=None):
    """T: dict of per-direction tables b, db, w (scaled), D, z."""
    kb, Bp = _arr3(T["b"])
    kdb, dBp = _arr3(T["db"])
    kw, Wp = _arr3(T["w"])
    kd, Dp = _arr3(T["D"])
    kz, Zp = _arr3(T["z"])
    out = np.zeros(nelmt * ncoeffs(shape, nm))
    d = None if diff is None else np.ascontiguousarray(diff, dtype=np.float64)
    lib().or_helmholtz(SHAPES[shape], int(deformed), nm, (ctypes.c_int * 3)(*nq), nelmt, Bp, dBp,
                       Wp, Dp, Zp, _p(np.ascontiguousarray(jac)), _p(np.ascontiguousarray(df)),
                       ctypes.c_double(lam), diff_mode, _p(d), _p(np.ascontiguousarray(x)),
                       _p(out))
    return out


class _HelmDesc(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int), ("deformed", ctypes.c_int), ("nm", ctypes.c_int),
                ("nq", ctypes.c_int * 3), ("nelmt", ctypes.c_int), ("B", _dp * 3),
                ("dB", _dp * 3), ("w", _dp * 3), ("D", _dp * 3), ("Z", _dp * 3),
                ("jac", _dp), ("df", _dp), ("lam", ctypes.c_double)]


def _helm_desc(shape, nm, nq, nelmt, T, jac, df, lam, deformed):
    keep = []
    d = _HelmDesc()
    d.shape, d.deformed, d.nm, d.nelmt = SHAPES[shape], int(deformed), nm, nelmt
    d.nq = (ctypes.c_int * 3)(*nq)
    for key, field in (("b", "B"), ("db", "dB"), ("w", "w"), ("D", "D"), ("z", "Z")):
        k, arr = _arr3(T[key])
        keep.append(k)
        setattr(d, field, arr)
    jac = np.ascontiguousarray(jac)
    df = np.ascontiguousarray(df)
    keep += [jac, df]
    d.jac, d.df, d.lam = _p(jac), _p(df), lam
    return d, keep


def helmholtz_diag(shape, nm, nq, nelmt, T, jac, df, lam=1.0, deformed=True):
    d, keep = _helm_desc(shape, nm, nq, nelmt, T, jac, df, lam, deformed)
    out = np.zeros(nelmt * ncoeffs(shape, nm))
    lib().or_helmholtz_diag(ctypes.byref(d), _p(out))
    return out


def pcg(shape, nm, nq, nelmt, T, jac, df, lam, deformed, nglob, ndir, gmap, sign, diag_inv,
        b_glob, tol=1e-10, maxit=5000):
    d, keep = _helm_desc(shape, nm, nq, nelmt, T, jac, df, lam, deformed)
    x = np.zeros(nglob)
    err = ctypes.c_double(0.0)
    gmap = np.ascontiguousarray(gmap, dtype=np.int32)
    its = lib().or_pcg(ctypes.byref(d), nglob, ndir, gmap.ctypes.data_as(_ip),
                       _p(None if sign is None else np.ascontiguousarray(sign)),
                       _p(np.ascontiguousarray(diag_inv)), _p(np.ascontiguousarray(b_glob)),
                       _p(x), ctypes.c_double(tol), maxit, ctypes.byref(err))
    return x, its, err.value


def assemble(gmap, sign, loc, nglob):
    out = np.zeros(nglob)
    np.add.at(out, gmap, loc if sign is None else sign * loc)
    return out


def global_to_local(gmap, sign, glob):
    v = glob[gmap]
    return v if sign is None else sign * v
