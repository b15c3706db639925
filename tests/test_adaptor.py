"""The C++ mirror of the Collections plugin interface
(nektar_b200/adaptor/nkb_collections.hpp) compiles against the C ABI and
behaves like the reference's operators: factory lookup by OperatorKey with
the new eB200 implementation type, NekError on failure."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests.helpers import ROOT, have_gpu

LIB_DIR = os.path.join(ROOT, "nektar_b200")


def _build(tmp_path):
    exe = str(tmp_path / "adaptor_demo")
    subprocess.check_call(["g++", "-std=c++17", "-O1", os.path.join(ROOT, "tests", "cpp",
                                                                     "adaptor_demo.cpp"),
                           "-L" + LIB_DIR, "-lnekb200", "-Wl,-rpath," + LIB_DIR, "-o", exe])
    return exe


def test_adaptor_compiles_and_reports_errors_as_nekerror(tmp_path):
    exe = _build(tmp_path)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    out = json.loads(p.stdout.strip().splitlines()[-1])
    if have_gpu():
        assert p.returncode == 0, p.stdout + p.stderr
    else:
        assert p.returncode == 3 and out["nekerror"] in (-7, -3), out
    # per-direction orders: refused with NKB_ERR_UNSUPPORTED before any device work
    assert out["per_direction_orders"] == -2, out


@pytest.mark.gpu
def test_adaptor_matches_c_abi(tmp_path):
    import nektar_b200 as nb
    exe = _build(tmp_path)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    out = json.loads(p.stdout.strip().splitlines()[-1])
    m = nb.BoxMesh("hex", 3, 5, 6, amp=0.05)
    op = nb.Operator("helmholtz", m)
    op.set_factors(1.5)
    x = np.sin(0.37 * np.arange(op.in_size))
    ny = float(np.sum(op(x) ** 2))
    assert abs(out["helmholtz_norm2"] - ny) <= 1e-12 * ny
    ipd = nb.Operator("iproduct_deriv", m)
    i = np.arange(ipd.in_size // 3)
    g = ipd.apply3(np.cos(0.11 * i), np.cos(0.11 * i + 1.0), np.cos(0.11 * i + 2.0))
    ng = float(np.sum(g ** 2))
    assert abs(out["iproduct_deriv_norm2"] - ng) <= 1e-12 * ng
    adr = nb.Operator("linear_adr", m)
    adr.set_factors(1.5)
    i = np.arange(m.nelmt * m.nt)
    adr.set_varcoeffs(1.0 + 0.1 * np.sin(0.05 * i), np.full(i.size, -0.5), 0.25 * np.cos(0.02 * i))
    na = float(np.sum(adr(x) ** 2))
    assert abs(out["linear_adr_norm2"] - na) <= 1e-12 * na
    assert out["dir_call_threw"] == 1
    assert out["cg_rel_residual"] < 1e-10 and out["cg_iterations"] > 0
