"""Build libnekb200.so in-tree with nvcc for sm_100a.

    python -m nektar_b200.build          # incremental
    python -m nektar_b200.build --force  # rebuild everything

The library is plain C ABI (include/nektar_b200.h); no torch headers are
involved. Objects go to nektar_b200/_build/, the shared library to
nektar_b200/libnekb200.so.
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnekb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC"]

SOURCES = ["nkb_setup.cpp", "nkb_ops.cu", "nkb_hex.cu", "nkb_hex_f64.cu", "nkb_hex_f32.cu",
           "nkb_cg.cu", "nkb_static.cu", "nkb_batch.cu", "nkb_dense.cu", "nkb_gen_f64.cu",
           "nkb_gen_f32.cu", "nkb_col_f64.cu", "nkb_col_f32.cu", "nkb_tc.cu", "nkb_sc.cu", "nkb_nccl.cpp",
           "nkb_geom.cu", "nkb_peak.cu"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "nektar_b200.h"))
    return hs


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= hdr_mtime):
            continue
        if src.endswith(".cu"):
            cmd = [nvcc] + NVCC_FLAGS + ["-c", path, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-I" + os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include"), "-c", path, "-o", obj]
        cmds.append(cmd)
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed = True
            sys.stderr.write(text)
        elif verbose and text.strip():
            sys.stderr.write(text)
    if failed:
        raise RuntimeError("nektar_b200 build failed")
    if force or cmds or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
