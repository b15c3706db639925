"""Shared helpers of the test suite (fixture loading, norms)."""
import glob
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference source tree (read-only; only CPU tests that read its session
# files use it), as oracle/Makefile's REFDIR
REFDIR = os.environ.get("REFDIR", "/root/reference")


def ref_path(rel):
    """A file of the reference tree by its path within the project."""
    return os.path.join(REFDIR, rel)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")




def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*_nm*_nq*_*.npz")))


def load_case(path):
    g = dict(np.load(path))
    name = os.path.basename(path)
    g["shape"] = name.split("_")[0]
    T = {k: [g["%s%d" % (k, d)] for d in range(3)] for k in ("b", "db", "w", "ws", "z", "D")}
    T["ptype"] = [int(p) for p in g["ptype"]]
    g["T"] = T
    return g


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
