"""The C-ABI shared library loads and exports every entry point that
include/nektar_b200.h declares; argument validation runs without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200 import _capi as C
from tests.helpers import ROOT, have_gpu

HEADER = os.path.join(ROOT, "include", "nektar_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nkb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = C.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(C.SIGNATURES), set(syms) ^ set(C.SIGNATURES)


def test_version_string():
    assert b"sm_100a" in C.lib().nkb_version()


def _desc(**kw):
    d = C.OpDesc()
    d.shape, d.optype, d.nm, d.nelmt = C.HEX, C.HELMHOLTZ, 3, 1
    d.nq = (ctypes.c_int * 3)(4, 4, 4)
    d.ptype = (ctypes.c_int * 3)(C.GLL, C.GLL, C.GLL)
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("kw,msg", [
    ({"shape": 3}, "unsupported shape"),
    ({"optype": 6}, "unsupported operator"),  # ePhysInterp1DScaled
    ({"nq": (ctypes.c_int * 3)(4, 4, 5)}, "not homogeneous"),
    ({"precision": 7}, "precision"),
    ({"nm": 1}, "out of range"),
])
def test_op_create_rejects_bad_descriptors(kw, msg):
    h = ctypes.c_void_p()
    rc = C.lib().nkb_op_create(ctypes.byref(_desc(**kw)), ctypes.byref(h))
    assert rc == C.NKB_ERR_INVALID
    assert msg in C.lib().nkb_last_error().decode()
    assert not h.value


def test_op_create_requires_tables():
    h = ctypes.c_void_p()
    rc = C.lib().nkb_op_create(ctypes.byref(_desc()), ctypes.byref(h))
    assert rc == C.NKB_ERR_INVALID and b"required" in C.lib().nkb_last_error()


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_no_device_is_reported_not_faked():
    m = nb.BoxMesh("hex", 1, 3, 4)
    with pytest.raises(nb.NektarB200Error) as e:
        nb.Operator("helmholtz", m)
    assert e.value.code in (C.NKB_ERR_NO_DEVICE, C.NKB_ERR_CUDA)


def test_points_rejects_unknown_type():
    z = np.zeros(4)
    assert C.lib().nkb_points(1, 4, z.ctypes.data_as(C.dp), z.ctypes.data_as(C.dp),
                              None) == C.NKB_ERR_UNSUPPORTED


@pytest.mark.parametrize("bm,im,msg", [
    ([0, 1, 1], [2], b"bm is not part"),
    ([0, 1], [1, 2], b"im is not part"),
    ([0, 4], [1, 2], b"bm is not part"),
    ([0, 1], [2, 3], b"bad arguments"),  # nb + ni != nc
])
def test_condense_rejects_index_lists_that_do_not_partition_the_modes(bm, im, msg):
    """The boundary / interior split is checked on the host before any
    device work (a dummy K pointer is never dereferenced)."""
    ip = ctypes.POINTER(ctypes.c_int)
    b = np.asarray(bm, dtype=np.int32)
    i = np.asarray(im, dtype=np.int32)
    dummy = ctypes.c_void_p(16)
    nc = len(bm) + len(im) - (msg == b"bad arguments")
    rc = C.lib().nkb_condense(4, nc, dummy, len(bm), b.ctypes.data_as(ip), len(im),
                              i.ctypes.data_as(ip), None, dummy, dummy, dummy, 0, None)
    assert rc == C.NKB_ERR_INVALID and msg in C.lib().nkb_last_error()
