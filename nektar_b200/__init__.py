"""nektar_b200: B200 (sm_100a) matrix-free spectral/hp element operators,
C0 assembly and Jacobi-preconditioned CG, behind the C ABI of
include/nektar_b200.h.

Python mirror of the reference's Collections operator interface
(Collections/Operator.h:137-245): an `Operator` is one collection of
same-shape elements; `GlobalLinSys` is GlobalLinSysIterativeFull with the
diagonal preconditioner. Arrays are numpy (host; copied in and out, the call
is synchronous like the reference's) or device pointers (torch tensors'
data_ptr(), stream ordered).
"""
import ctypes

import numpy as np

from . import _capi as C
from ._capi import (BWDTRANS, DEVICE_PTRS, DIFF_CONST, DIFF_NONE, DIFF_VAR, FP32, FP64, GLL,
                    HELMHOLTZ, HEX, HOST_PTRS, IPRODUCT, IPRODUCT_DERIV, LINEAR_ADR, MODIFIED_A, MODIFIED_B, MODIFIED_C,
                    PHYSDERIV, PRISM, RADAU_A1, RADAU_A2, TET, NektarB200Error, check)

SHAPES = {"hex": HEX, "prism": PRISM, "tet": TET}
OPTYPES = {"bwdtrans": BWDTRANS, "helmholtz": HELMHOLTZ, "linear_adr": LINEAR_ADR,
           "iproduct": IPRODUCT,
           "iproduct_deriv": IPRODUCT_DERIV, "physderiv": PHYSDERIV}
WEIGHT_FACTOR = {GLL: 1.0, RADAU_A1: 0.5, RADAU_A2: 0.25}

__all__ = ["Operator", "GlobalLinSys", "BoxMesh", "points", "basis", "shape_tables", "lib",
           "NektarB200Error", "SHAPES", "OPTYPES"]


def lib():
    return C.lib()


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def points(ptype, n):
    """z, raw weights w and column-major D of a points type (GaussPoints)."""
    z, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
    check(lib().nkb_points(ptype, n, _dp(z), _dp(w), _dp(D)))
    return z, w, D


def basis(btype, nm, z, D):
    """bdata, dbdata of a modified basis (Basis::GenBasis layout)."""
    n = len(z)
    nb = {MODIFIED_A: nm, MODIFIED_B: nm * (nm + 1) // 2,
          MODIFIED_C: nm * (nm + 1) * (nm + 2) // 6}[btype]
    b, db = np.zeros(nb * n), np.zeros(nb * n)
    rc = lib().nkb_basis(btype, nm, n, _dp(_f64(z)), _dp(_f64(D)), _dp(b), _dp(db))
    if rc < 0:
        check(rc)
    return b, db


def shape_spec(shape, nq0):
    """(basis type, points type, npoints) per direction for a 3-D shape, as
    Nektar sets them up (SpatialDomains/MeshGraph.cpp:1709-1750): GLL in the
    Cartesian directions, Gauss-Radau alpha=1 / alpha=2 in collapsed ones."""
    if shape == "hex":
        return [(MODIFIED_A, GLL, nq0)] * 3
    if shape == "prism":
        return [(MODIFIED_A, GLL, nq0), (MODIFIED_A, GLL, nq0), (MODIFIED_B, RADAU_A1, nq0 - 1)]
    if shape == "tet":
        return [(MODIFIED_A, GLL, nq0), (MODIFIED_B, RADAU_A1, nq0 - 1),
                (MODIFIED_C, RADAU_A2, nq0 - 1)]
    raise ValueError(shape)


def ncoeffs(shape, nm):
    if shape == "hex":
        return nm ** 3
    if shape == "prism":
        return nm * nm * (nm + 1) // 2
    return nm * (nm + 1) * (nm + 2) // 6


def shape_tables(shape, nm, nq0):
    """1-D tables of a shape: dict with per-direction lists b, db, w (raw),
    ws (Radau-scaled, as MatrixFree SetUpZW), z, D, ptype; and nq."""
    T = {"b": [], "db": [], "w": [], "ws": [], "z": [], "D": [], "ptype": []}
    nq = []
    for bt, pt, n in shape_spec(shape, nq0):
        z, w, D = points(pt, n)
        b, db = basis(bt, nm, z, D)
        for k, v in (("b", b), ("db", db), ("w", w), ("ws", w * WEIGHT_FACTOR[pt]), ("z", z),
                     ("D", D), ("ptype", pt)):
            T[k].append(v)
        nq.append(n)
    return T, tuple(nq)


class BoxMesh:
    """Unit-cube box of n^3 cells (hexes, or 2 prisms / 6 tets per cell),
    optionally curved by x' = x + amp sin(pi x) sin(pi y) sin(pi z), with
    analytic geometric factors at the quadrature points (Collections layout)."""

    def __init__(self, shape, n, nm, nq0, amp=0.0, deformed=None, cells=None, coords=False,
                 geom_device=None):
        """geom_device: a CUDA device index to compute jac / df (and xyz) on
        that device (torch tensors, nkb_geom_fill_device) instead of the host
        (numpy arrays, nkb_geom_fill)."""
        self.shape, self.n, self.nm, self.amp = shape, n, nm, amp
        self.deformed = bool(amp != 0.0) if deformed is None else bool(deformed)
        self.T, self.nq = shape_tables(shape, nm, nq0)
        self.nt = self.nq[0] * self.nq[1] * self.nq[2]
        self.nc = ncoeffs(shape, nm)
        self.cells = None if cells is None else np.ascontiguousarray(cells, dtype=np.int32)
        req = C.GeomRequest()
        req.shape, req.n, req.amp = SHAPES[shape], n, amp
        req.ncells = 0 if self.cells is None else len(self.cells)
        req.cells = None if self.cells is None else self.cells.ctypes.data_as(C.ip)
        req.nq = (ctypes.c_int * 3)(*self.nq)
        self._z = [_f64(z) for z in self.T["z"]]
        req.z = (C.dp * 3)(*[_dp(z) for z in self._z])
        req.deformed = int(self.deformed)
        self.nelmt = int(lib().nkb_geom_nelmt(ctypes.byref(req)))
        ncol = self.nelmt * self.nt if self.deformed else self.nelmt
        if geom_device is not None:
            import torch
            dev = "cuda:%d" % geom_device
            self.jac = torch.empty(ncol, dtype=torch.float64, device=dev)
            self.df = torch.empty((9, ncol), dtype=torch.float64, device=dev)
            self.xyz = (torch.empty((3, self.nelmt * self.nt), dtype=torch.float64, device=dev)
                        if coords else None)
            check(lib().nkb_geom_fill_device(
                ctypes.byref(req), self.jac.data_ptr(), self.df.data_ptr(),
                None if self.xyz is None else self.xyz.data_ptr(), geom_device, None))
            return
        self.jac = np.zeros(ncol)
        self.df = np.zeros((9, ncol))
        self.xyz = np.zeros((3, self.nelmt * self.nt)) if coords else None
        check(lib().nkb_geom_fill(ctypes.byref(req), _dp(self.jac), _dp(self.df),
                                  _dp(self.xyz)))

    def assembly(self):
        """(map, nglob, ndir) of the hex box's C0 numbering, Dirichlet first."""
        if self.shape != "hex" or self.cells is not None:
            raise ValueError("assembly maps are built for full hex boxes")
        gmap = np.zeros(self.nelmt * self.nc, dtype=np.int32)
        nglob, ndir = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().nkb_hex_box_assembly(self.n, self.nm, gmap.ctypes.data_as(C.ip),
                                         ctypes.byref(nglob), ctypes.byref(ndir)))
        return gmap, nglob.value, ndir.value


class Operator:
    """One collection operator (Collections::Operator) on the device."""

    def __init__(self, optype, mesh=None, *, shape=None, nm=None, nq=None, nelmt=None, T=None,
                 jac=None, df=None, deformed=None, precision="fp64", device=0):
        if mesh is not None:
            shape, nm, nq, nelmt, T = mesh.shape, mesh.nm, mesh.nq, mesh.nelmt, mesh.T
            jac, df, deformed = mesh.jac, mesh.df, mesh.deformed
        self.optype = OPTYPES[optype] if isinstance(optype, str) else optype
        self.shape, self.nm, self.nq, self.nelmt = shape, nm, tuple(nq), nelmt
        self.precision = FP64 if precision in ("fp64", FP64) else FP32
        self._keep = []
        d = C.OpDesc()
        d.shape, d.optype, d.nm = SHAPES[shape], self.optype, nm
        d.nq = (ctypes.c_int * 3)(*nq)
        d.ptype = (ctypes.c_int * 3)(*T["ptype"])
        d.nelmt, d.deformed = nelmt, int(bool(deformed))

        def arr3(key):
            arrs = [_f64(a) for a in T[key]]
            self._keep.extend(arrs)
            return (C.dp * 3)(*[_dp(a) for a in arrs])

        d.bdata, d.w, d.z, d.D = arr3("b"), arr3("w"), arr3("z"), arr3("D")

        def geom(a):
            # a CUDA tensor (FP64, contiguous) stays on the device: its
            # address is passed and the library copies device to device
            if hasattr(a, "is_cuda") and a.is_cuda:
                if str(a.dtype) != "torch.float64" or not a.is_contiguous():
                    raise ValueError("device geometry must be contiguous FP64")
                self._keep.append(a)
                return ctypes.cast(ctypes.c_void_p(a.data_ptr()), C.dp)
            a = _f64(a)
            self._keep.append(a)
            return _dp(a)

        if jac is not None:
            d.jac = geom(jac)
        if df is not None:
            d.df = geom(df)
        d.precision, d.device = self.precision, device
        h = ctypes.c_void_p()
        check(lib().nkb_op_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self._keep = []
        nin, nout = ctypes.c_long(), ctypes.c_long()
        check(lib().nkb_op_sizes(self.h, ctypes.byref(nin), ctypes.byref(nout)))
        self.in_size, self.out_size = nin.value, nout.value

    def set_factors(self, lam=1.0, diff_mode=DIFF_NONE, diff=None):
        """Helmholtz_MatrixFree::UpdateFactors: lambda and diffusion tensor
        (LinearADR: lambda only; the operator applies -lambda)."""
        d = None if diff is None else _f64(diff)
        check(lib().nkb_op_set_factors(self.h, float(lam), diff_mode, _dp(d)))
        self.lam = float(lam)

    def set_varcoeffs(self, velx, vely, velz):
        """LinearADR advection velocities (UpdateVarcoeffs): host arrays of
        nelmt * ntot values, or device pointers (ints)."""
        if all(isinstance(v, int) for v in (velx, vely, velz)):
            check(lib().nkb_op_set_varcoeffs(self.h, velx, vely, velz, DEVICE_PTRS))
            return
        vs = [_f64(v) for v in (velx, vely, velz)]
        check(lib().nkb_op_set_varcoeffs(self.h, *[v.ctypes.data for v in vs], HOST_PTRS))

    def __call__(self, x):
        """Host arrays in, host arrays out (synchronous)."""
        x = _f64(x)
        if x.size != self.in_size:
            raise ValueError("input size %d != %d" % (x.size, self.in_size))
        nout = 3 if self.optype == PHYSDERIV else 1
        outs = [np.zeros(self.out_size) for _ in range(nout)] + [None] * (3 - nout)
        check(lib().nkb_op_apply(self.h, x.ctypes.data, *[None if o is None else o.ctypes.data
                                                           for o in outs], HOST_PTRS, None))
        return tuple(outs[:nout]) if nout > 1 else outs[0]

    def apply3(self, f0, f1, f2):
        """IProductWRTDerivBase with the vector field as three host arrays
        (IProductWRTDerivBase_MatrixFree::operator(), synchronous)."""
        fs = [_f64(f) for f in (f0, f1, f2)]
        n = self.in_size // 3
        if self.optype != IPRODUCT_DERIV or any(f.size != n for f in fs):
            raise ValueError("apply3 takes three fields of %d values of an iproduct_deriv "
                             "operator" % n)
        out = np.zeros(self.out_size)
        check(lib().nkb_op_apply3(self.h, *[f.ctypes.data for f in fs], out.ctypes.data,
                                  HOST_PTRS, None))
        return out

    def apply3_device(self, f0_ptr, f1_ptr, f2_ptr, out_ptr, stream=None):
        """apply3 on device pointers, stream-ordered."""
        check(lib().nkb_op_apply3(self.h, f0_ptr, f1_ptr, f2_ptr, out_ptr, DEVICE_PTRS, stream))

    def apply_device(self, x_ptr, out0, out1=None, out2=None, stream=None):
        """Device pointers (ints); stream-ordered on `stream` (cudaStream_t int)."""
        fn = lib().nkb_op_apply if self.precision == FP64 else lib().nkb_op_apply_f32
        if self.precision == FP64:
            check(fn(self.h, x_ptr, out0, out1, out2, DEVICE_PTRS, stream))
        else:
            check(fn(self.h, x_ptr, out0, out1, out2, stream))

    def kernel(self, gather=False):
        """Name of the device kernel the operator runs (autotuned choice)."""
        return lib().nkb_op_kernel(self.h, int(bool(gather))).decode()

    def last_kernel_ms(self):
        ms = ctypes.c_float()
        check(lib().nkb_op_last_kernel_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def check_error(self):
        """Raise if a bounded wait inside one of the operator's kernels gave
        up since the last check (device-pointer applies; host applies and
        solves check by themselves)."""
        check(lib().nkb_op_check_error(self.h))

    def set_wait_limit(self, polls):
        """Test hook: polls after which the kernels' bounded waits give up
        (0: at once; negative: the default)."""
        check(lib().nkb_op_set_wait_limit(self.h, int(polls)))

    def helmholtz_diag(self):
        out = np.zeros(self.nelmt * ncoeffs(self.shape, self.nm))
        check(lib().nkb_op_helmholtz_diag(self.h, out.ctypes.data, HOST_PTRS, None))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().nkb_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many collections' operators of one type applied in one call
    (ExpList::GeneralMatrixOp over the collections), concurrently on the
    device. in/out: concatenated per-collection local vectors."""

    def __init__(self, ops, nstreams=4):
        self.ops = list(ops)
        self.precision = self.ops[0].precision
        handles = (ctypes.c_void_p * len(self.ops))(*[o.h.value for o in self.ops])
        h = ctypes.c_void_p()
        check(lib().nkb_batch_create(handles, len(self.ops), int(nstreams), ctypes.byref(h)))
        self.h = h
        nin, nout = ctypes.c_long(), ctypes.c_long()
        check(lib().nkb_batch_sizes(self.h, ctypes.byref(nin), ctypes.byref(nout)))
        self.in_size, self.out_size = nin.value, nout.value

    def __call__(self, x):
        """Host arrays in and out (copies inside the call)."""
        x = _f64(x)
        if x.size != self.in_size:
            raise ValueError("batch input has %d values, expected %d" % (x.size, self.in_size))
        y = np.zeros(self.out_size)
        check(lib().nkb_batch_apply(self.h, x.ctypes.data, y.ctypes.data, HOST_PTRS, None))
        return y

    def apply_device(self, x_ptr, y_ptr, stream=None):
        """Device pointers; FP64 or FP32 per the operators' precision."""
        if self.precision == FP32:
            check(lib().nkb_batch_apply_f32(self.h, x_ptr, y_ptr, stream))
        else:
            check(lib().nkb_batch_apply(self.h, x_ptr, y_ptr, DEVICE_PTRS, stream))

    def last_ms(self):
        ms = ctypes.c_float(0.0)
        check(lib().nkb_batch_last_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().nkb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DenseOperator:
    """Per-element dense operator y_e = M_e x_e (nkb_op_create_dense[_rect]):
    mats (nelmt, rows, cols) FP64, e.g. the Schur complements of static
    condensation. Square ones are usable wherever a Helmholtz Operator is
    (GlobalLinSys, apply)."""

    def __init__(self, mats, device=0):
        mats = np.ascontiguousarray(mats, dtype=np.float64)
        self.nelmt, rows, cols = mats.shape
        self.n, self.rows, self.cols = cols, rows, cols
        self.precision, self.optype = FP64, C.DENSE_BLOCK
        h = ctypes.c_void_p()
        check(lib().nkb_op_create_dense_rect(rows, cols, self.nelmt, mats.ctypes.data, device,
                                             ctypes.byref(h)))
        self.h = h
        self.in_size, self.out_size = self.nelmt * cols, self.nelmt * rows

    @classmethod
    def from_device(cls, mats, device=0):
        """The same from a (nelmt, rows, cols) FP64 device tensor (copied on
        the device; the tensor may be freed afterwards)."""
        self = object.__new__(cls)
        self.nelmt, rows, cols = (int(v) for v in mats.shape)
        self.n, self.rows, self.cols = cols, rows, cols
        self.precision, self.optype = FP64, C.DENSE_BLOCK
        h = ctypes.c_void_p()
        check(lib().nkb_op_create_dense_rect(rows, cols, self.nelmt, ctypes.c_void_p(mats.data_ptr()),
                                             device, ctypes.byref(h)))
        self.h = h
        self.in_size, self.out_size = self.nelmt * cols, self.nelmt * rows
        return self

    def __call__(self, x):
        x = _f64(x)
        if x.size != self.in_size:
            raise ValueError("input size %d != %d" % (x.size, self.in_size))
        y = np.zeros(self.out_size)
        check(lib().nkb_op_apply(self.h, x.ctypes.data, y.ctypes.data, None, None, HOST_PTRS,
                                 None))
        return y

    def apply_device(self, x_ptr, y_ptr, stream=None):
        check(lib().nkb_op_apply(self.h, x_ptr, y_ptr, None, None, DEVICE_PTRS, stream))

    def kernel(self, gather=False):
        return lib().nkb_op_kernel(self.h, int(bool(gather))).decode()

    def last_kernel_ms(self):
        ms = ctypes.c_float()
        check(lib().nkb_op_last_kernel_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().nkb_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GlobalLinSys:
    """GlobalLinSysIterativeFull + PreconditionerDiagonal + NekLinSysIterCG."""

    def __init__(self, ops, gmap, nglob, ndir, sign=None, device=0, ops32=None):
        """ops: FP64 Helmholtz operators in local-space order; ops32: optional
        FP32 twins (same meshes) enabling the mixed-precision solve."""
        self.ops = list(ops)
        self.ops32 = None if ops32 is None else list(ops32)
        self.nloc = int(sum(o.in_size for o in self.ops))
        self.nglob, self.ndir = int(nglob), int(ndir)
        gmap = np.ascontiguousarray(gmap, dtype=np.int32)
        sign = None if sign is None else _f64(sign)
        handles = (ctypes.c_void_p * len(self.ops))(*[o.h.value for o in self.ops])
        d = C.SysDesc()
        h32 = None
        if self.ops32 is not None:
            h32 = (ctypes.c_void_p * len(self.ops32))(*[o.h.value for o in self.ops32])
        d.nops, d.ops, d.ops32 = len(self.ops), handles, h32
        d.nloc, d.nglob, d.ndir = self.nloc, self.nglob, self.ndir
        d.map = gmap.ctypes.data_as(C.ip)
        d.sign = _dp(sign)
        d.device = device
        h = ctypes.c_void_p()
        check(lib().nkb_sys_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h

    @staticmethod
    def _opts(tol, maxit, check_interval, use_graph, mixed=False, inner_tol=0.0, max_outer=0):
        o = C.CGOpts()
        o.tol, o.maxit, o.check_interval, o.use_graph = tol, maxit, check_interval, int(use_graph)
        o.mixed, o.inner_tol, o.max_outer = int(bool(mixed)), inner_tol, max_outer
        return o

    def solve(self, b_loc, x_loc=None, tol=1e-9, maxit=5000, check_interval=16, use_graph=True,
              raise_on_maxit=True, mixed=False, inner_tol=0.0, max_outer=0):
        """Host arrays: local rhs and local Dirichlet values -> local solution.
        mixed=True: FP32 CG with FP64 reliable updates (inner_tol = FP32
        residual reduction between updates, max_outer = maximum updates)."""
        b = _f64(b_loc)
        x = np.zeros(self.nloc) if x_loc is None else _f64(x_loc).copy()
        rep = C.CGReport()
        opts = self._opts(tol, maxit, check_interval, use_graph, mixed, inner_tol, max_outer)
        rc = lib().nkb_cg_solve(self.h, b.ctypes.data, x.ctypes.data, ctypes.byref(opts),
                                ctypes.byref(rep), HOST_PTRS, None)
        if rc != C.NKB_OK and (raise_on_maxit or rc != C.NKB_ERR_NOT_CONVERGED):
            check(rc)
        return x, rep

    def solve_device(self, b_ptr, x_ptr, tol=1e-9, maxit=5000, check_interval=16,
                     use_graph=True, stream=None, mixed=False, inner_tol=0.0, max_outer=0):
        rep = C.CGReport()
        opts = self._opts(tol, maxit, check_interval, use_graph, mixed, inner_tol, max_outer)
        check(lib().nkb_cg_solve(self.h, b_ptr, x_ptr, ctypes.byref(opts), ctypes.byref(rep),
                                 DEVICE_PTRS, stream))
        return rep

    def solve_host_ptrs(self, b_ptr, x_ptr, tol=1e-9, maxit=5000, check_interval=16,
                        use_graph=True, stream=None, mixed=False, inner_tol=0.0, max_outer=0):
        """Host (ideally pinned) buffers by address: copies in and out inside
        the call, on `stream`."""
        rep = C.CGReport()
        opts = self._opts(tol, maxit, check_interval, use_graph, mixed, inner_tol, max_outer)
        check(lib().nkb_cg_solve(self.h, b_ptr, x_ptr, ctypes.byref(opts), ctypes.byref(rep),
                                 HOST_PTRS, stream))
        return rep

    # ---- non-blocking solve, clones, per-system lambda (serving layer) ----
    def begin(self, b_ptr, x_ptr, tol=1e-9, maxit=5000, check_interval=16, use_graph=True,
              stream=None, mixed=False, inner_tol=0.0, max_outer=0):
        """Start a solve on device buffers and return at once; drive it with
        poll() until it reports done, then end()."""
        self._opts_keep = self._opts(tol, maxit, check_interval, use_graph, mixed, inner_tol,
                                     max_outer)
        check(lib().nkb_cg_begin(self.h, b_ptr, x_ptr, ctypes.byref(self._opts_keep),
                                 DEVICE_PTRS, stream))

    def poll(self, wait=False):
        """Advance the solve by at most one block of device work; True once done."""
        done = ctypes.c_int(0)
        check(lib().nkb_cg_poll(self.h, int(bool(wait)), ctypes.byref(done)))
        return bool(done.value)

    def end(self, raise_on_maxit=True):
        rep = C.CGReport()
        rc = lib().nkb_cg_end(self.h, ctypes.byref(rep))
        if rc != C.NKB_OK and (raise_on_maxit or rc != C.NKB_ERR_NOT_CONVERGED):
            check(rc)
        return rep

    def clone(self):
        """Another system over the same operators, map and diagonal, with its
        own vectors and stream."""
        c = object.__new__(GlobalLinSys)
        c.ops, c.ops32 = self.ops, self.ops32
        c.nloc, c.nglob, c.ndir = self.nloc, self.nglob, self.ndir
        h = ctypes.c_void_p()
        check(lib().nkb_sys_clone(self.h, ctypes.byref(h)))
        c.h = h
        return c

    def set_lambda(self, lam):
        """Helmholtz lambda of this system's solves (overrides the operators')."""
        check(lib().nkb_sys_set_lambda(self.h, float(lam)))

    def set_blocks(self, blocks):
        """Block-Jacobi preconditioner (nkb_sys_set_blocks): a list of
        (dofs, inverse) pairs, dofs the global indices (>= ndir) of one block
        and inverse its n x n inverse. Dofs outside every block keep Jacobi."""
        idx = [np.asarray(d, dtype=np.int64) - self.ndir for d, _ in blocks]
        ptr = np.zeros(len(blocks) + 1, dtype=np.int32)
        ptr[1:] = np.cumsum([i.size for i in idx])
        bidx = np.ascontiguousarray(np.concatenate(idx), dtype=np.int32)
        binv = np.concatenate([np.asarray(m, dtype=np.float64).T.ravel() for _, m in blocks])
        check(lib().nkb_sys_set_blocks(self.h, len(blocks), ptr.ctypes.data_as(C.ip),
                                       bidx.ctypes.data_as(C.ip), _dp(binv)))

    def set_block_inverses(self, bptr, dofs, binv_ptr):
        """Block-Jacobi preconditioner from inverses already in device memory
        (nkb_blocks_invert's layout): bptr the block pointers, dofs the
        blocks' global dofs (>= ndir) one block after another, binv_ptr the
        device address of the inverses (copied)."""
        bptr = np.ascontiguousarray(bptr, dtype=np.int32)
        bidx = np.ascontiguousarray(np.asarray(dofs, dtype=np.int64) - self.ndir, dtype=np.int32)
        check(lib().nkb_sys_set_blocks(self.h, bptr.size - 1, bptr.ctypes.data_as(C.ip),
                                       bidx.ctypes.data_as(C.ip),
                                       ctypes.cast(ctypes.c_void_p(binv_ptr), C.dp)))

    def footprint(self):
        """(shared bytes, instance bytes) of device memory held by the system."""
        a, b = ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(lib().nkb_sys_footprint(self.h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def profile(self, iters=20):
        """Per-kernel device time of one CG iteration (CUDA events)."""
        p = C.SysProfile()
        check(lib().nkb_sys_profile_iteration(self.h, iters, ctypes.byref(p)))
        return {k: getattr(p, k) for k, _ in C.SysProfile._fields_}

    def diag_inv(self):
        out = np.zeros(self.nglob - self.ndir)
        check(lib().nkb_sys_diag_inv(self.h, out.ctypes.data, HOST_PTRS, None))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().nkb_sys_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
