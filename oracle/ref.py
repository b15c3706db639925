"""Test infrastructure only (the oracle): ctypes loader for the reference's own
MatrixFreeOps kernels compiled in place into oracle/_ref/libnkref_<isa>.so by
oracle/Makefile (see oracle/ref_harness.cpp and oracle/ref_common.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's reference / cpu_baseline
legs use this module; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# numbering as LibUtilities::ShapeType / Collections::OperatorType / PointsType / BasisType
SHAPES = {"tet": 5, "prism": 7, "hex": 8}
OPS = {"bwdtrans": 0, "helmholtz": 1, "linear_adr": 2, "iproduct": 3, "iproduct_deriv": 4,
       "physderiv": 5}
GLL, RADAU_A1, RADAU_A2 = 4, 11, 12
MOD_A, MOD_B, MOD_C = 4, 5, 6

_lib = None
_isa = None


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def best_isa():
    fl = _cpu_flags()
    if {"avx512f", "avx512dq", "avx512vl"} <= fl:
        return "avx512"
    if {"avx2", "fma"} <= fl:
        return "avx2"
    return "scalar"


def physical_cpus():
    """One logical CPU per physical core among those this process may run
    on (sysfs topology; every allowed CPU when the topology is unreadable)."""
    allowed = sorted(os.sched_getaffinity(0))
    seen, out = set(), []
    for c in allowed:
        base = "/sys/devices/system/cpu/cpu%d/topology/" % c
        try:
            with open(base + "core_id") as f:
                core = f.read().strip()
            with open(base + "physical_package_id") as f:
                pkg = f.read().strip()
        except OSError:
            return allowed
        if (pkg, core) not in seen:
            seen.add((pkg, core))
            out.append(c)
    return out


def set_cpus(cpus):
    """Pin the reference driver's worker thread t to cpus[t % len(cpus)]
    (empty: no pinning)."""
    arr = (ctypes.c_int * max(len(cpus), 1))(*cpus)
    lib().nkref_set_cpus(len(cpus), arr)


def available():
    return os.path.exists(os.path.join(REF_DIR, "libnkref_%s.so" % best_isa()))


def lib(isa=None):
    """Load (once) the widest reference build this CPU can run."""
    global _lib, _isa
    isa = isa or best_isa()
    if _lib is not None and _isa == isa:
        return _lib
    path = os.path.join(REF_DIR, "libnkref_%s.so" % isa)
    if not os.path.exists(path):
        raise FileNotFoundError("reference kernels not built: %s (run make -C oracle ref)" % path)
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    vp = ctypes.c_void_p
    for s in SHAPES:
        f = getattr(L, "nkref_%s_create" % s)
        f.restype = vp
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int,
                      ctypes.POINTER(dp), ctypes.POINTER(dp), ctypes.POINTER(dp),
                      ctypes.POINTER(dp), ctypes.POINTER(dp), dp, dp, ctypes.c_int]
        f = getattr(L, "nkref_%s_set_factors" % s)
        f.restype = None
        f.argtypes = [vp, ctypes.c_double, ctypes.c_int, dp, ctypes.c_int]
        f = getattr(L, "nkref_%s_set_adr" % s)
        f.restype = None
        f.argtypes = [vp, ctypes.c_double, dp]
        f = getattr(L, "nkref_%s_apply" % s)
        f.restype = None
        f.argtypes = [vp, dp, dp, dp, dp]
        f = getattr(L, "nkref_%s_destroy" % s)
        f.restype = None
        f.argtypes = [vp]
        getattr(L, "nkref_%s_simd_width" % s).restype = ctypes.c_int
    L.nkref_points.restype = ctypes.c_int
    L.nkref_points.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.nkref_basis.restype = ctypes.c_int
    L.nkref_basis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp]
    L.nkref_weight_factor.restype = ctypes.c_double
    L.nkref_weight_factor.argtypes = [ctypes.c_int]
    L.nkref_set_cpus.restype = None
    L.nkref_set_cpus.argtypes = [ctypes.c_int, ip]
    L.nkref_pcg_solve.restype = ctypes.c_int
    L.nkref_pcg_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ip, dp, ip,
                                  ctypes.POINTER(ctypes.c_long), vp, vp, dp, dp, dp,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    _lib, _isa = L, isa
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def points(ptype, np_):
    L = lib()
    z = np.zeros(np_)
    w = np.zeros(np_)
    D = np.zeros(np_ * np_)
    if L.nkref_points(ptype, np_, _dp(z), _dp(w), _dp(D)) != 0:
        raise ValueError("unsupported points type %d" % ptype)
    return z, w, D


def nbasis(btype, nm):
    return {MOD_A: nm, MOD_B: nm * (nm + 1) // 2, MOD_C: nm * (nm + 1) * (nm + 2) // 6}[btype]


def basis(btype, nm, ptype, np_):
    z, w, D = points(ptype, np_)
    nb = nbasis(btype, nm)
    b = np.zeros(nb * np_)
    db = np.zeros(nb * np_)
    lib().nkref_basis(btype, nm, np_, _dp(z), _dp(D), _dp(b), _dp(db))
    return b, db


def weight_factor(ptype):
    return lib().nkref_weight_factor(ptype)


class RefOp:
    """One reference MatrixFree operator over a collection of elements.

    tables: dict with per-direction lists 'b', 'db', 'w' (already scaled as
    Operator.hpp SetUpZW), 'z', 'D'. jac/df in CoalescedGeomData layout.
    """

    def __init__(self, shape, op, nm, nq, nelmt, tables, jac=None, df=None, deformed=False,
                 nthreads=1):
        self.L = lib()
        self.shape = shape
        self.op = OPS[op] if isinstance(op, str) else op
        self._keep = []

        def arr3(key):
            vals = tables.get(key)
            if vals is None:
                return None
            arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in vals]
            self._keep.extend(arrs)
            return (ctypes.POINTER(ctypes.c_double) * 3)(*[_dp(a) for a in arrs])

        nqa = (ctypes.c_int * 3)(*nq)
        self.jac = None if jac is None else np.ascontiguousarray(jac, dtype=np.float64)
        self.df = None if df is None else np.ascontiguousarray(df, dtype=np.float64)
        self.nm, self.nq, self.nelmt = nm, tuple(nq), nelmt
        self.h = getattr(self.L, "nkref_%s_create" % shape)(
            self.op, int(deformed), nm, nqa, nelmt, arr3("b"), arr3("db"), arr3("w"), arr3("z"),
            arr3("D"), None if self.jac is None else _dp(self.jac),
            None if self.df is None else _dp(self.df), nthreads)
        self._apply = getattr(self.L, "nkref_%s_apply" % shape)
        self._apply_ptr = ctypes.cast(self._apply, ctypes.c_void_p)

    def set_factors(self, lam=1.0, const_diff=None, var_diff=None):
        d = np.zeros(6)
        isc = isv = 0
        if const_diff is not None:
            d[:] = const_diff
            isc = 1
        if var_diff is not None:
            d[:] = var_diff
            isv = 1
        getattr(self.L, "nkref_%s_set_factors" % self.shape)(self.h, float(lam), isc, _dp(d), isv)

    def set_adr(self, lam, vel):
        """LinearADR factors as the Collections operator takes them: lambda
        and the three velocity fields (3 * nelmt * nt values)."""
        self._vel = np.ascontiguousarray(vel, dtype=np.float64)
        getattr(self.L, "nkref_%s_set_adr" % self.shape)(self.h, float(lam), _dp(self._vel))

    def apply(self, x, out0, out1=None, out2=None):
        self._apply(self.h, _dp(x), _dp(out0), None if out1 is None else _dp(out1),
                    None if out2 is None else _dp(out2))

    def __del__(self):
        try:
            getattr(self.L, "nkref_%s_destroy" % self.shape)(self.h)
        except Exception:
            pass


def pcg_solve(nglob, ndir, gmap, sign, asm_ptr, asm_idx, op, diag_inv, b_glob, tol=1e-10,
              maxit=5000, nthreads=1, max_iters_to_run=0):
    """CPU PCG of NekLinSysIterCG driving the reference Helmholtz kernels."""
    L = lib()
    x = np.zeros(nglob)
    err = np.zeros(1)
    ip = ctypes.POINTER(ctypes.c_int)
    its = L.nkref_pcg_solve(
        nglob, ndir, len(gmap), gmap.ctypes.data_as(ip),
        None if sign is None else _dp(sign), asm_ptr.ctypes.data_as(ip),
        asm_idx.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), op._apply_ptr, op.h,
        _dp(diag_inv), _dp(b_glob), _dp(x), tol, maxit, nthreads, max_iters_to_run, _dp(err))
    return x, its, float(err[0])


def tables(shape, nm, nq0):
    """Reference tables (reference Polylib + restated GenBasis) with weights
    scaled as MatrixFree SetUpZW scales them, and the point counts."""
    spec = {"hex": [(MOD_A, GLL, 0)] * 3,
            "prism": [(MOD_A, GLL, 0), (MOD_A, GLL, 0), (MOD_B, RADAU_A1, -1)],
            "tet": [(MOD_A, GLL, 0), (MOD_B, RADAU_A1, -1), (MOD_C, RADAU_A2, -1)]}[shape]
    T = {"b": [], "db": [], "w": [], "z": [], "D": []}
    nq = []
    for bt, pt, dq in spec:
        n = nq0 + dq
        z, w, D = points(pt, n)
        b, db = basis(bt, nm, pt, n)
        for k, v in (("b", b), ("db", db), ("w", w * weight_factor(pt)), ("z", z), ("D", D)):
            T[k].append(v)
        nq.append(n)
    return T, tuple(nq)


def helmholtz_diag(op, ncoef):
    """Diagonal of every element's Helmholtz matrix with the reference
    kernels: apply the operator to the m-th unit vector of all elements at
    once, for every m (the reference assembles it from dense element
    matrices, PreconditionerDiagonal.cpp:93-125)."""
    ne = op.nelmt
    x = np.zeros(ne * ncoef)
    y = np.zeros(ne * ncoef)
    out = np.zeros(ne * ncoef)
    for m in range(ncoef):
        x[m::ncoef] = 1.0
        op.apply(x, y)
        out[m::ncoef] = y[m::ncoef]
        x[m::ncoef] = 0.0
    return out
