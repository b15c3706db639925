"""ctypes declarations of the C ABI in include/nektar_b200.h.

The product path has no CPU fallback: importing this module raises if
libnekb200.so has not been built (python -m nektar_b200.build).
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnekb200.so")

c_int, c_long, c_double, c_float = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_float
c_void_p, c_char_p, c_size_t = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t
P = ctypes.POINTER
dp, fp, ip = P(c_double), P(c_float), P(c_int)

# status codes
NKB_OK = 0
NKB_ERR_INVALID = -1
NKB_ERR_UNSUPPORTED = -2
NKB_ERR_CUDA = -3
NKB_ERR_NOMEM = -4
NKB_ERR_NOT_CONVERGED = -5
NKB_ERR_NONFINITE = -6
NKB_ERR_NO_DEVICE = -7
NKB_ERR_TIMEOUT = -8

TET, PRISM, HEX = 5, 7, 8
BWDTRANS, HELMHOLTZ, LINEAR_ADR, IPRODUCT, IPRODUCT_DERIV, PHYSDERIV = 0, 1, 2, 3, 4, 5
DENSE_BLOCK = 64
GLL, RADAU_A1, RADAU_A2 = 4, 11, 12
MODIFIED_A, MODIFIED_B, MODIFIED_C = 4, 5, 6
FP64, FP32 = 0, 1
DEVICE_PTRS, HOST_PTRS = 0, 1
DIFF_NONE, DIFF_CONST, DIFF_VAR = 0, 1, 2


class OpDesc(ctypes.Structure):
    _fields_ = [("shape", c_int), ("optype", c_int), ("nm", c_int), ("nq", c_int * 3),
                ("ptype", c_int * 3), ("nelmt", c_int), ("deformed", c_int),
                ("bdata", dp * 3), ("w", dp * 3), ("z", dp * 3), ("D", dp * 3),
                ("jac", dp), ("df", dp), ("precision", c_int), ("device", c_int)]


class SysDesc(ctypes.Structure):
    _fields_ = [("nops", c_int), ("ops", P(c_void_p)), ("ops32", P(c_void_p)), ("nloc", c_long),
                ("nglob", c_int), ("ndir", c_int), ("map", ip), ("sign", dp), ("device", c_int)]


class CGOpts(ctypes.Structure):
    _fields_ = [("tol", c_double), ("maxit", c_int), ("check_interval", c_int),
                ("use_graph", c_int), ("mixed", c_int), ("inner_tol", c_double),
                ("max_outer", c_int)]


class CGReport(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("outer_iterations", c_int), ("rel_residual", c_double),
                ("converged", c_int), ("device_ms", c_double), ("kernel_launches", c_long),
                ("restarts", c_int)]


class ShardPlan(ctypes.Structure):
    _fields_ = [("rank", c_int), ("nint", c_int), ("nown", c_int),
                ("dir_owned", P(ctypes.c_ubyte)), ("nshared", c_int), ("shared", ip),
                ("sptr", ip), ("ssrc", ip), ("nnbr", c_int), ("nbr", ip), ("nptr", ip),
                ("nidx", ip)]


class SysProfile(ctypes.Structure):
    _fields_ = [("op_ms", c_double), ("assemble_ms", c_double), ("update_ms", c_double),
                ("scalars_ms", c_double), ("op_bytes", c_double), ("op_flops", c_double)]


class GeomRequest(ctypes.Structure):
    _fields_ = [("shape", c_int), ("n", c_int), ("amp", c_double), ("ncells", c_int),
                ("cells", ip), ("nq", c_int * 3), ("z", dp * 3), ("deformed", c_int)]


# every symbol the header declares, with its signature
SIGNATURES = {
    "nkb_last_error": (c_char_p, []),
    "nkb_version": (c_char_p, []),
    "nkb_points": (c_int, [c_int, c_int, dp, dp, dp]),
    "nkb_basis": (c_int, [c_int, c_int, c_int, dp, dp, dp, dp]),
    "nkb_op_create": (c_int, [P(OpDesc), P(c_void_p)]),
    "nkb_op_set_factors": (c_int, [c_void_p, c_double, c_int, dp]),
    "nkb_op_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_op_apply_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "nkb_op_apply_host_static": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                         c_void_p]),
    "nkb_op_create_dense": (c_int, [c_int, c_int, c_void_p, c_int, P(c_void_p)]),
    "nkb_op_create_dense_rect": (c_int, [c_int, c_int, c_int, c_void_p, c_int, P(c_void_p)]),
    "nkb_op_set_varcoeffs": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "nkb_op_apply3": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_op_sizes": (c_int, [c_void_p, P(c_long), P(c_long)]),
    "nkb_op_helmholtz_diag": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_op_last_kernel_ms": (c_int, [c_void_p, P(c_float)]),
    "nkb_op_check_error": (c_int, [c_void_p]),
    "nkb_condense": (c_int, [c_int, c_int, c_void_p, c_int, ip, c_int, ip, dp, c_void_p, c_void_p,
                             c_void_p, c_int, c_void_p]),
    "nkb_tc_selftest": (c_int, [c_int, c_int, c_int, fp, fp, fp, P(ctypes.c_uint)]),
    "nkb_blocks_accumulate": (c_int, [c_int, ip, c_int, ip, ip, ip, P(ctypes.c_byte), c_int, c_int,
                                      c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_blocks_invert": (c_int, [c_int, ip, c_void_p, c_int, c_void_p]),
    "nkb_op_set_wait_limit": (c_int, [c_void_p, c_int]),
    "nkb_op_destroy": (None, [c_void_p]),
    "nkb_op_kernel": (c_char_p, [c_void_p, c_int]),
    "nkb_sys_create": (c_int, [P(SysDesc), P(c_void_p)]),
    "nkb_cg_solve": (c_int, [c_void_p, c_void_p, c_void_p, P(CGOpts), P(CGReport), c_int,
                             c_void_p]),
    "nkb_sys_assemble": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "nkb_sys_global_to_local": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "nkb_sys_matvec_local": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "nkb_sys_diag_inv": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_sys_profile_iteration": (c_int, [c_void_p, c_int, P(SysProfile)]),
    "nkb_sys_destroy": (None, [c_void_p]),
    "nkb_comm_unique_id": (c_int, [P(ctypes.c_ubyte)]),
    "nkb_comm_create": (c_int, [P(ctypes.c_ubyte), c_int, c_int, c_int, P(c_void_p)]),
    "nkb_comm_destroy": (None, [c_void_p]),
    "nkb_shard_group_create": (c_int, [P(c_void_p), P(ShardPlan), c_int, c_void_p,
                                       P(c_void_p)]),
    "nkb_shard_group_solve": (c_int, [c_void_p, P(c_void_p), P(c_void_p), P(CGOpts),
                                      P(CGReport), c_int]),
    "nkb_shard_group_destroy": (None, [c_void_p]),
    "nkb_batch_create": (c_int, [P(c_void_p), c_int, c_int, P(c_void_p)]),
    "nkb_batch_sizes": (c_int, [c_void_p, P(c_long), P(c_long)]),
    "nkb_batch_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_batch_apply_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "nkb_batch_last_ms": (c_int, [c_void_p, P(c_float)]),
    "nkb_batch_destroy": (None, [c_void_p]),
    "nkb_cg_begin": (c_int, [c_void_p, c_void_p, c_void_p, P(CGOpts), c_int, c_void_p]),
    "nkb_cg_poll": (c_int, [c_void_p, c_int, P(c_int)]),
    "nkb_cg_end": (c_int, [c_void_p, P(CGReport)]),
    "nkb_sys_clone": (c_int, [c_void_p, P(c_void_p)]),
    "nkb_sys_set_lambda": (c_int, [c_void_p, c_double]),
    "nkb_sys_set_blocks": (c_int, [c_void_p, c_int, ip, ip, dp]),
    "nkb_op_element_matrices": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "nkb_sys_footprint": (c_int, [c_void_p, P(c_size_t), P(c_size_t)]),
    "nkb_geom_nelmt": (c_long, [P(GeomRequest)]),
    "nkb_geom_fill": (c_int, [P(GeomRequest), dp, dp, dp]),
    "nkb_peak_probe": (c_int, [c_int, c_int, dp]),
    "nkb_geom_fill_device": (c_int, [P(GeomRequest), c_void_p, c_void_p, c_void_p, c_int,
                                     c_void_p]),
    "nkb_hex_box_assembly": (c_int, [c_int, c_int, ip, ip, ip]),
}

_lib = None


class NektarB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("nektar_b200 error %d: %s" % (code, msg))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libnekb200.so is not built (%s); run python -m nektar_b200.build"
                              % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != NKB_OK:
        raise NektarB200Error(rc, lib().nkb_last_error().decode(errors="replace"))
    return rc
