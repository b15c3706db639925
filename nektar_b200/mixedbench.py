"""Mixed-element benchmark: element Helmholtz on a 40^3 box grid whose cells
are, by a seeded permutation, 20000 hexes, 15000 cells split into 2 prisms
each and 10000 cells split into 6 tets each (110000 elements), P drawn in
{2..10} per cell, curved by the box map, coefficients uniform in [-1, 1].
One collection per (shape, P), all applied by one batched call.

    python -m nektar_b200.mixedbench [--iters 10] [--cpu] [--precision fp32]

Prints one JSON line: local GDOF/s of the batched apply (device time, CUDA
events), the same collections applied one after another on one stream, the
algorithmic bytes and their fraction of the measured HBM bandwidth, and with
--cpu the reference kernels (oracle/_ref) applied collection by collection on
all host cores.
"""
import argparse
import json
import os
import time

import numpy as np


def measure(n=40, cells=(20000, 15000, 10000), pmin=2, pmax=10, iters=10, warmup=3, streams=4,
            cpu=False, precision="fp64", groups_detail=True, device=0):
    """The C4 measurement as a dict (see the module docstring)."""
    import torch

    import nektar_b200 as nb
    from nektar_b200.mixed_mesh import MixedMesh

    mm = MixedMesh(n, tuple(cells), pmin, pmax, amp=0.05, seed=0)
    ops, groups, cpu_s, cpu_threads = [], [], 0.0, None
    t_setup = time.perf_counter()
    for (shape, p, _cells), m in zip(mm.groups, mm.meshes()):
        op = nb.Operator("helmholtz", m, precision=precision, device=device)
        op.set_factors(1.0)
        ops.append(op)
        esz = 8 if precision == "fp64" else 4
        groups.append({"shape": shape, "P": p, "elements": m.nelmt, "dofs": m.nelmt * m.nc,
                       "bytes": m.nelmt * esz * (7 * m.nt + 2 * m.nc)})
        if cpu:
            from oracle import ref
            cpu_threads = len(os.sched_getaffinity(0))
            T, nq = ref.tables(shape, p + 1, p + 2)
            R = ref.RefOp(shape, "helmholtz", p + 1, nq, m.nelmt, T, jac=m.jac, df=m.df,
                          deformed=True, nthreads=cpu_threads)
            R.set_factors(1.0)
            x = np.random.default_rng(p).uniform(-1, 1, m.nelmt * m.nc)
            y = np.zeros_like(x)
            R.apply(x, y)
            t0 = time.perf_counter()
            R.apply(x, y)
            cpu_s += time.perf_counter() - t0
            del R
        m.jac = m.df = None
    t_setup = time.perf_counter() - t_setup
    B = nb.Batch(ops, nstreams=streams)
    dofs = sum(g["dofs"] for g in groups)
    byts = sum(g["bytes"] for g in groups)
    dt = torch.float64 if precision == "fp64" else torch.float32
    esz = 8 if precision == "fp64" else 4
    dv = "cuda:%d" % device
    x = torch.rand(B.in_size, dtype=dt, device=dv) * 2 - 1
    y = torch.empty(B.out_size, dtype=dt, device=dv)
    s = torch.cuda.Stream(device=device)
    torch.cuda.synchronize()

    def timed(fn):
        for _ in range(warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(iters):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / iters

    ms_batch = timed(lambda: B.apply_device(x.data_ptr(), y.data_ptr(), stream=s.cuda_stream))
    offs_in = np.cumsum([0] + [op.in_size for op in ops])
    offs_out = np.cumsum([0] + [op.out_size for op in ops])

    def sequential():
        for k, op in enumerate(ops):
            op.apply_device(x.data_ptr() + esz * int(offs_in[k]),
                            y.data_ptr() + esz * int(offs_out[k]), stream=s.cuda_stream)

    ms_seq = timed(sequential)
    if groups_detail:
        # each collection alone (same stream, same buffers)
        for k, op in enumerate(ops):
            groups[k]["ms"] = timed(lambda k=k, op=op: op.apply_device(
                x.data_ptr() + esz * int(offs_in[k]), y.data_ptr() + esz * int(offs_out[k]),
                stream=s.cuda_stream))
            groups[k]["gb_s"] = groups[k]["bytes"] / groups[k]["ms"] / 1e6
            groups[k]["kernel"] = op.kernel()
    peaks = {}
    try:
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    out = {
        "metric": "mixed-element Helmholtz apply, local GDOF/s",
        "workload": "%d^3 grid: %d hex cells, %d cells -> 2 prisms, %d cells -> 6 tets, P %d..%d "
                    "per cell, curved" % (n, *cells, pmin, pmax),
        "elements": int(sum(g["elements"] for g in groups)), "collections": len(groups),
        "precision": precision, "local_dofs": int(dofs), "algorithmic_bytes": int(byts),
        "batched": {"ms": ms_batch, "gdof_s": dofs / ms_batch / 1e6,
                    "gb_s": byts / ms_batch / 1e6, "hbm_frac": byts / ms_batch / 1e6 / hbm,
                    "streams": streams},
        "sequential": {"ms": ms_seq, "gdof_s": dofs / ms_seq / 1e6},
        "setup_s": t_setup,
    }
    if groups_detail:
        out["groups"] = groups
    if cpu:
        out["cpu_reference"] = {"ms": cpu_s * 1e3, "gdof_s": dofs / cpu_s / 1e9,
                                "threads": cpu_threads, "kind": "reference",
                                "sample": "one apply of every collection (after one warm-up)"}
    B.close()
    for op in ops:
        op.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=40)
    ap.add_argument("--cells", type=int, nargs=3, default=(20000, 15000, 10000))
    ap.add_argument("--pmin", type=int, default=2)
    ap.add_argument("--pmax", type=int, default=10)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--cpu", action="store_true", help="time the reference CPU kernels too")
    ap.add_argument("--precision", default="fp64", choices=("fp64", "fp32"))
    a = ap.parse_args()
    out = measure(a.n, a.cells, a.pmin, a.pmax, a.iters, a.warmup, a.streams, a.cpu, a.precision)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
