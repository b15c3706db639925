"""Micro-benchmark of one element operator on a curved box (device-resident
input, CUDA-event timing), used for profiling captures:

    python -m nektar_b200.opbench --op helmholtz --shape hex --n 24 --p 6 --iters 20

--op matvec times the pieces of one CG iteration of the assembled system
instead (element Helmholtz with the local<-global gather fused, assemble,
vector update, scalars), FP64.
"""
import argparse
import json

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="helmholtz")
    ap.add_argument("--shape", default="hex")
    ap.add_argument("--n", type=int, default=24)
    ap.add_argument("--p", type=int, default=6)
    ap.add_argument("--amp", type=float, default=0.05)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--iters", type=int, default=20)
    a = ap.parse_args()
    import torch

    import nektar_b200 as nb
    nm = a.p + 1
    m = nb.BoxMesh(a.shape, a.n, nm, nm + 1, amp=a.amp)
    if a.op == "matvec":
        gmap, nglob, ndir = m.assembly()
        op = nb.Operator("helmholtz", m)
        op.set_factors(1.0)
        S = nb.GlobalLinSys([op], gmap, nglob, ndir)
        S.profile(iters=max(a.warmup, 1))
        prof = S.profile(iters=a.iters)
        print(json.dumps({"op": "matvec", "shape": a.shape, "n": a.n, "P": a.p,
                          "nelmt": m.nelmt, "nglob": nglob, **prof,
                          "op_GB_s": prof["op_bytes"] / prof["op_ms"] / 1e6}))
        return
    op = nb.Operator(a.op, m, precision=a.precision)
    if a.op == "linear_adr":
        op.set_factors(1.0)
        i = np.arange(m.nelmt * m.nt)
        op.set_varcoeffs(np.sin(0.01 * i), np.cos(0.01 * i), np.full(i.size, 0.5))
    dt = torch.float64 if a.precision == "fp64" else torch.float32
    x = torch.rand(op.in_size, dtype=dt, device="cuda")
    outs = [torch.empty(op.out_size, dtype=dt, device="cuda")
            for _ in range(3 if a.op == "physderiv" else 1)]
    ptrs = [o.data_ptr() for o in outs] + [None] * (3 - len(outs))
    s = torch.cuda.Stream()
    for _ in range(a.warmup):
        op.apply_device(x.data_ptr(), *ptrs, stream=s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.iters):
        op.apply_device(x.data_ptr(), *ptrs, stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.iters
    ncomp = {"helmholtz": 7, "linear_adr": 10, "physderiv": 9, "iproduct_deriv": 9,
             "iproduct": 1, "bwdtrans": 0}[a.op]
    esz = 8 if a.precision == "fp64" else 4
    byts = m.nelmt * esz * (ncomp * m.nt + (op.in_size + len(outs) * op.out_size) / m.nelmt)
    print(json.dumps({"op": a.op, "shape": a.shape, "n": a.n, "P": a.p, "nelmt": m.nelmt,
                      "precision": a.precision, "kernel": op.kernel(), "ms": ms,
                      "GB_s": byts / ms / 1e6, "GDOF_s": m.nelmt * m.nc / ms / 1e6}))


if __name__ == "__main__":
    main()
