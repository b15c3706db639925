#!/usr/bin/env python
"""Benchmark of the B200 matrix-free Helmholtz path.

Workload (one GPU): the full FP64 Helmholtz solve  -lap u + lambda u = f  on
32^3 curved hexes (x' = x + 0.05 sin(pi x) sin(pi y) sin(pi z) in every
coordinate), P = 6 (7 modes), Q = 8 GLL points per direction, lambda = 1,
matrix-free PCG with the Jacobi (diagonal) preconditioner to a relative
residual of 1e-10, manufactured solution u = sin(pi x) sin(pi y) sin(pi z)
(zero Dirichlet data). A step is one complete solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0): CG solves/s over all GPUs, device-timed with
CUDA events (max over ranks), plus the end-to-end figure through the public
API with host buffers, the roofline of the dominant kernel (the element
Helmholtz operator), the reference CPU baseline and the SM clocks seen
during the timed region. With N > 1 (torchrun) every rank solves its own
copy: the solve does not shard, so the GPUs run replicas.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Helmholtz CG solves/s (FP64, PCG+Jacobi, rel. residual 1e-10)"
AMP, LAM, TOL = 0.05, 1.0, 1e-10
# FP32-residual reduction between the mixed solve's FP64 reliable updates. Measured at
# equal accuracy (1e-10 of the converged FP64 solution) against FP64: 24^3 P=8 1.24x,
# 1.26x, 1.38x, 1.24x and 32^3 P=6 1.548x, 1.552x, 1.541x, 1.486x at 0.05, 0.1, 0.25,
# 0.5 (at 0.25 the P=8 solve restarts its FP32 recurrence once instead of twice)
MIXED_INNER_TOL = 0.25
# the default is the 32^3, P=6 solve; 24^3 at P=8 is the higher-order
# companion (same map, same criterion)
WORKLOADS = {
    "hex32_p6": (32, 7, "fp64 Helmholtz solve, 32^3 curved hex, P=6 Q=8, PCG+Jacobi to 1e-10"),
    "hex24_p8": (24, 9, "fp64 Helmholtz solve, 24^3 curved hex, P=8 Q=10, PCG+Jacobi to 1e-10"),
}
N_CELLS, NM, WORKLOAD = WORKLOADS["hex32_p6"]
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the headline solve (no parity, mixed, P=8, operator and "
                         "mixed-element keys)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="hex32_p6")
    ap.add_argument("--shard", action="store_true",
                    help="one solve sharded over the N GPUs by element partition (strong "
                         "scaling; NCCL exchange of the shared dofs) instead of N replicas")
    args = ap.parse_args()
    global N_CELLS, NM, WORKLOAD
    N_CELLS, NM, WORKLOAD = WORKLOADS[args.workload]
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": FALLBACK_HBM_GBS}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_record(tag):
    """The reference CPU path's recorded full solve of a workload (iterations,
    residual, error, tight-tolerance figures; tests/golden/make_c2_reference.py)
    and its solution digest, or None."""
    path = os.path.join(ROOT, "tests", "golden", "%s_reference_cg.json" % tag)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        rec = json.load(f)
    dpath = os.path.join(ROOT, "tests", "golden", "%s_reference_solution.npz" % tag)
    if os.path.exists(dpath):
        with np.load(dpath) as z:
            rec["digest"] = {k: z[k] for k in z.files}
    return rec


WORKLOAD_TAG = {"hex32_p6": "c2", "hex24_p8": "c3"}


def reference_iterations():
    """The reference's recorded solve of the current workload (None if not
    recorded: the caller scales by the FP64 device solve's count, the same
    algorithm and criterion)."""
    for name, (n, nm, _) in WORKLOADS.items():
        if (n, nm) == (N_CELLS, NM):
            return reference_record(WORKLOAD_TAG[name])
    return None


ITERS_PER_BLOCK = 200  # contiguous CG iterations per timed CPU block


def workload_config(nelmt, nloc, nglob, ndir, world=1):
    """The workload's config dict, shared by both arms."""
    return {"workload": WORKLOAD, "elements": nelmt, "P": NM - 1, "Q": NM + 1, "nloc": nloc,
            "nglob": nglob, "ndir": ndir, "lambda": LAM, "tol": TOL,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "no flush: the operator streams the geometry (%.2f GB per matvec, > 126 MB L2)"
                  % (nelmt * 7 * (NM + 1) ** 3 * 8 / 1e9)}


class ReferenceCPU:
    """The reference CPU path on the host cores: the reference's MatrixFreeOps
    kernels (oracle/_ref, built from the reference sources) driven by the
    restated NekLinSysIterCG + AssemblyMapCG loop with the Jacobi
    preconditioner of PreconditionerDiagonal (diagonal from the reference
    kernels), one worker thread pinned to each physical core. The same
    routine gives the reference arm and the b200 arm's cpu_baseline."""

    def __init__(self):
        from oracle import mesh as OM
        from oracle import ref
        self.ref = ref
        self.cpus = ref.physical_cpus()
        ref.set_cpus(self.cpus)
        self.nthreads = len(self.cpus)
        t0 = time.perf_counter()
        T, nq = ref.tables("hex", NM, NM + 1)
        jac, df, xyz = OM.hex_box_geometry(N_CELLS, T["z"][0], AMP)
        self.ne, self.nc = N_CELLS ** 3, NM ** 3
        self.op = ref.RefOp("hex", "helmholtz", NM, nq, self.ne, T, jac=jac, df=df,
                            deformed=True, nthreads=self.nthreads)
        self.op.set_factors(LAM)
        ipo = ref.RefOp("hex", "iproduct", NM, nq, self.ne, T, jac=jac, deformed=True,
                        nthreads=self.nthreads)
        u = np.sin(np.pi * xyz[0]) * np.sin(np.pi * xyz[1]) * np.sin(np.pi * xyz[2])
        del jac, df, xyz
        b_loc = np.zeros(self.ne * self.nc)
        ipo.apply((3 * np.pi ** 2 + LAM) * u, b_loc)
        del ipo, u
        self.gmap, self.nglob, self.ndir = OM.hex_box_assembly(N_CELLS, NM)
        self.aptr, self.aidx = OM.csr_from_map(self.gmap, self.nglob)
        self.b_glob = np.bincount(self.gmap, weights=b_loc, minlength=self.nglob)
        # PreconditionerDiagonal: element diagonals from the reference kernels
        dloc = ref.helmholtz_diag(self.op, self.nc)
        self.dinv = 1.0 / np.bincount(self.gmap, weights=dloc,
                                      minlength=self.nglob)[self.ndir:]
        self.setup_s = time.perf_counter() - t0
        self.rec = reference_iterations()

    def block(self, iters):
        """Seconds per iteration of one contiguous block of `iters` CG
        iterations of the solve (from its start: fresh vectors)."""
        t0 = time.perf_counter()
        _, its, _ = self.ref.pcg_solve(self.nglob, self.ndir, self.gmap, None, self.aptr,
                                       self.aidx, self.op, self.dinv, self.b_glob, tol=1e-30,
                                       maxit=10 ** 6, nthreads=self.nthreads,
                                       max_iters_to_run=iters)
        dt = time.perf_counter() - t0
        return dt / max(its, 1), dt

    def iterations_per_solve(self, fallback=None):
        return self.rec["iterations"] if self.rec else fallback

    def measure(self, nblocks, iters_per_solve, iters=ITERS_PER_BLOCK):
        """Median over nblocks blocks; solves/s from the median seconds per
        iteration and the iterations a solve takes."""
        per, secs = [], []
        for _ in range(nblocks):
            p, dt = self.block(iters)
            per.append(p)
            secs.append(dt)
        med = statistics.median(per)
        return {"value": 1.0 / (med * iters_per_solve), "unit": "solves/s",
                "cores": self.nthreads, "kind": "reference",
                "sample": "%d blocks of %d contiguous CG iterations of the full workload "
                          "(%d threads, one per physical core, pinned), solves/s = 1 / "
                          "(median seconds per iteration x %d iterations per solve)"
                          % (nblocks, iters, self.nthreads, iters_per_solve),
                "seconds_per_iteration": {"min": min(per), "median": med, "max": max(per)},
                "block_seconds": secs, "iterations_per_solve": iters_per_solve,
                "setup_seconds": self.setup_s, "cpu": cpu_model(), "simd": self.ref.best_isa(),
                "preconditioner": "Jacobi (reference kernels' element diagonals)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference kernels not built (make -C oracle ref)"}))
        return
    R = ReferenceCPU()
    if R.rec is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference CG iteration count is recorded for hex32_p6 and "
                          "hex24_p8 only; the b200 arm's cpu_baseline covers %s"
                          % args.workload}))
        return
    for _ in range(max(args.warmup, 0)):
        R.block(10)
    base = R.measure(max(args.steps, 1), R.iterations_per_solve())
    value = base["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(base["block_seconds"]),
        "step": "one contiguous block of %d CG iterations of the %d-iteration solve"
                % (ITERS_PER_BLOCK, R.iterations_per_solve()),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (manufactured solution, zero Dirichlet data)",
        "config": workload_config(R.ne, R.ne * R.nc, R.nglob, R.ndir, world),
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ACC_TARGET = 1e-10  # relative L2 error against the converged FP64 solution
TOL_LADDER = (1e-11, 5e-12, 2e-12, 1e-12, 5e-13, 2e-13, 1e-13)
TOL_CONVERGED = 1e-14
K_CHECK = 32


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Problem:
    """One curved-box Helmholtz solve on the device: FP64 and FP32 operators,
    the system, the manufactured right-hand side, device and pinned buffers."""

    def __init__(self, nb, torch, n, nm, dev, coords=True):
        self.n, self.nm, self.dev = n, nm, dev
        self.mesh = nb.BoxMesh("hex", n, nm, nm + 1, amp=AMP, coords=coords)
        self.gmap, self.nglob, self.ndir = self.mesh.assembly()
        self.op = nb.Operator("helmholtz", self.mesh, device=dev)
        self.op.set_factors(LAM)
        self.op32 = nb.Operator("helmholtz", self.mesh, device=dev, precision="fp32")
        self.op32.set_factors(LAM)
        self.S = nb.GlobalLinSys([self.op], self.gmap, self.nglob, self.ndir, device=dev,
                                 ops32=[self.op32])
        x, y, z = self.mesh.xyz
        self.u = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        ipo = nb.Operator("iproduct", self.mesh, device=dev)
        self.b_host = ipo((3 * np.pi ** 2 + LAM) * self.u)
        ipo.close()
        self.mesh.xyz = self.mesh.jac = self.mesh.df = None
        self.nloc = self.mesh.nelmt * self.mesh.nc
        self.stream = torch.cuda.Stream(device=dev)
        self.sp = self.stream.cuda_stream
        self.torch = torch
        self.b_dev = torch.tensor(self.b_host, device=f"cuda:{dev}")
        self.x_dev = torch.zeros(self.nloc, dtype=torch.float64, device=f"cuda:{dev}")

    def solve(self, tol=TOL, mixed=False):
        with self.torch.cuda.stream(self.stream):
            self.x_dev.zero_()
        return self.S.solve_device(self.b_dev.data_ptr(), self.x_dev.data_ptr(), tol=tol,
                                   maxit=20000, check_interval=K_CHECK, stream=self.sp,
                                   mixed=mixed, inner_tol=MIXED_INNER_TOL)

    def x(self):
        self.torch.cuda.synchronize()
        return self.x_dev.cpu().numpy()

    def timed(self, steps, tol=TOL, mixed=False):
        """steps solves back to back, CUDA events on the solve stream: (ms, reports)."""
        torch = self.torch
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(self.stream)
        reps = [self.solve(tol, mixed) for _ in range(steps)]
        e1.record(self.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), reps

    def rms_vs_exact(self, nb, xl):
        """RMS error of the solution against the exact one at the quadrature points."""
        bwd = nb.Operator("bwdtrans", self.mesh, device=self.dev)
        rms = float(np.sqrt(np.mean((bwd(xl) - self.u) ** 2)))
        bwd.close()
        return rms

    def close(self):
        self.S.close()
        self.op.close()
        self.op32.close()


def equal_accuracy(P, steps, x_conv):
    """FP64 and mixed-precision solves/s at the same accuracy: each path runs
    at the loosest residual tolerance of TOL_LADDER whose solution is within
    ACC_TARGET (relative L2) of the converged FP64 solution (chosen on untimed
    solves), then `steps` timed solves at that tolerance."""
    out = {}
    for name, mixed in (("fp64", False), ("mixed", True)):
        tol, err = TOL_LADDER[-1], None
        for t in TOL_LADDER:
            P.solve(t, mixed)
            err = _rel(P.x(), x_conv)
            if err <= ACC_TARGET:
                tol = t
                break
        ms, reps = P.timed(steps, tol, mixed)
        err = _rel(P.x(), x_conv)
        r = reps[-1]
        out[name] = {"value": 1e3 * steps / ms, "unit": "solves/s", "tol": tol,
                     "rel_l2_vs_fp64_converged": err, "iterations": r.iterations,
                     "latency_ms": {"p50": float(np.percentile([q.device_ms for q in reps], 50)),
                                    "p99": float(np.percentile([q.device_ms for q in reps], 99))}}
        if mixed:
            out[name].update({"reliable_updates": r.outer_iterations, "restarts": r.restarts})
    return out


def mixed_block(P, steps, x_conv, fp64_value):
    """The mixed-precision result object: equal-accuracy comparison and the
    mixed solve at the headline residual criterion."""
    acc = equal_accuracy(P, steps, x_conv)
    m = acc["mixed"]
    ms, reps = P.timed(steps, TOL, True)
    x_m = P.x()
    return {
        "metric": "solves/s at %g relative L2 error against the converged FP64 solution "
                  "(residual %g)" % (ACC_TARGET, TOL_CONVERGED),
        "value": m["value"], "unit": "solves/s", "tol": m["tol"],
        "rel_l2_vs_fp64_solution": m["rel_l2_vs_fp64_converged"],
        "fp64_at_same_accuracy": acc["fp64"],
        "speedup_vs_fp64": m["value"] / acc["fp64"]["value"],
        "iterations": m["iterations"], "reliable_updates": m["reliable_updates"],
        "restarts": m["restarts"], "latency_ms": m["latency_ms"],
        "at_headline_residual": {"value": 1e3 * steps / ms, "tol": TOL,
                                 "speedup_vs_fp64_headline": 1e3 * steps / ms / fp64_value,
                                 "rel_l2_vs_fp64_converged": _rel(x_m, x_conv),
                                 "fp32_iterations": reps[-1].iterations},
        "fp32_operator": P.op32.kernel(gather=True),
        "scheme": "FP32 PCG (FP32 operators, vectors, Jacobi; FP64 dot sums) with FP64 reliable "
                  "updates: true residual b - Ax recomputed with the FP64 operator each time the "
                  "FP32 residual drops by %g; stop on the FP64 residual" % MIXED_INNER_TOL,
    }


def digest_check(rec, xl, x_conv):
    """Distance of the device solutions from the reference CPU path's recorded
    solutions at the digest positions (tests/golden/make_c2_reference.py)."""
    if not rec or "digest" not in rec:
        return None
    d = rec["digest"]
    pos = d["positions"]
    return {"iterations_reference": rec["iterations"],
            "rms_error_vs_exact_reference": rec["rms_error_vs_exact"],
            "rel_l2_vs_reference_solution": _rel(xl[pos], d["x"]),
            "converged_rel_l2_vs_reference_converged": _rel(x_conv[pos], d["x_tight"]),
            "positions": int(pos.size)}


def compute_peaks(nb, dev):
    """The device's FP64 FMA, FP64 tensor-core MMA and FP32 FMA rates in
    TFLOP/s, measured in place (nkb_peak_probe); None where unmeasurable."""
    import ctypes
    out = {}
    for kind, key in ((0, "fp64_fma_tflops"), (1, "fp64_mma_tflops"), (2, "fp32_fma_tflops")):
        v = ctypes.c_double(0.0)
        rc = nb.lib().nkb_peak_probe(kind, dev, ctypes.byref(v))
        out[key] = v.value if rc == 0 else None
    return out


def hex_flops(nm, nq):
    """Algorithmic FLOPs of one Hex Helmholtz element (sum factorisation:
    BwdTrans and one inner product, the collocation gradient and its
    transpose, the metric and the mass term)."""
    return (4 * (nq * nm ** 3 + nq ** 2 * nm ** 2 + nq ** 3 * nm) + 12 * nq ** 4
            + 18 * nq ** 3)


def operator_roofline(nb, torch, dev, n, p, precision, hbm, iters=20, peaks=None):
    """Element Helmholtz apply on an n^3 curved box at order p (local
    vectors, autotuned kernel): ms, GB/s of the algorithmic bytes, fraction;
    with peaks, TFLOP/s of the algorithmic FLOPs and their fraction of the
    precision's measured rate (FP64: the higher of FMA and tensor-core MMA)."""
    nm = p + 1
    m = nb.BoxMesh("hex", n, nm, nm + 1, amp=AMP)
    op = nb.Operator("helmholtz", m, device=dev, precision=precision)
    op.set_factors(LAM)
    dt = torch.float64 if precision == "fp64" else torch.float32
    esz = 8 if precision == "fp64" else 4
    x = torch.rand(op.in_size, dtype=dt, device=f"cuda:{dev}")
    y = torch.empty(op.out_size, dtype=dt, device=f"cuda:{dev}")
    s = torch.cuda.Stream(device=dev)
    for _ in range(3):
        op.apply_device(x.data_ptr(), y.data_ptr(), stream=s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(iters):
        op.apply_device(x.data_ptr(), y.data_ptr(), stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / iters
    byts = m.nelmt * esz * (7 * m.nt + 2 * m.nc)
    out = {"mesh": "%d^3" % n, "P": p, "precision": precision, "kernel": op.kernel(), "ms": ms,
           "gb_s": byts / ms / 1e6, "frac": byts / ms / 1e6 / hbm,
           "algorithmic_bytes": byts}
    flops = m.nelmt * hex_flops(nm, nm + 1)
    out["algorithmic_flops"] = flops
    out["tflops"] = flops / (ms * 1e-3) / 1e12
    if peaks:
        pk = (max(v for v in (peaks.get("fp64_fma_tflops"), peaks.get("fp64_mma_tflops")) if v)
              if precision == "fp64" else peaks.get("fp32_fma_tflops"))
        if pk:
            out["compute_frac"] = out["tflops"] / pk
    op.close()
    return out


def run_b200(args, rank, world, local):
    import torch
    import nektar_b200 as nb

    from nektar_b200 import replicas
    torch.cuda.set_device(local)
    dev = local
    pg = replicas.init(world, local, "nccl")
    peaks, peak_src = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))

    # the reference CPU path first, in a process that holds no device or
    # pinned memory yet (the same routine and blocks as the reference arm)
    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                R = ReferenceCPU()
                rec0 = reference_iterations()
                if rec0 is None:
                    cpu_base = {"value": None, "unavailable": "no recorded reference solve"}
                else:
                    cpu_base = R.measure(3, R.iterations_per_solve())
                del R
            else:
                cpu_base = {"value": None, "unavailable": "reference kernels not built"}
        except Exception as exc:  # the baseline must never sink the GPU number
            cpu_base = {"value": None, "unavailable": repr(exc)[:200]}

    peaks_c = compute_peaks(nb, dev)
    P = Problem(nb, torch, N_CELLS, NM, dev)
    nloc, nglob, ndir = P.nloc, P.nglob, P.ndir
    b_pin = torch.tensor(P.b_host).pin_memory()
    x_pin = torch.zeros(nloc, dtype=torch.float64).pin_memory()
    S = P.S

    for _ in range(max(args.warmup, 3)):
        P.solve()
    torch.cuda.synchronize()

    def barrier():
        replicas.barrier(pg)

    # ---- timed region: K device-resident solves -----------------------------
    with ClockSampler(dev) as clocks:
        barrier()
        ms, reps = P.timed(args.steps)
        barrier()
    lat = [r.device_ms for r in reps]
    ms_max = replicas.max_over_ranks(ms, pg, f"cuda:{dev}")
    value = replicas.whole_job_rate(args.steps, world, ms_max)
    x_fp64 = P.x()

    # ---- end to end: public API with pinned host buffers -----------------------
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(P.stream)
    for _ in range(args.steps):
        x_pin.zero_()
        S.solve_host_ptrs(b_pin.data_ptr(), x_pin.data_ptr(), tol=TOL, check_interval=K_CHECK,
                          stream=P.sp)
    e1.record(P.stream)
    torch.cuda.synchronize()
    e2e = replicas.whole_job_rate(
        args.steps, world, replicas.max_over_ranks(e0.elapsed_time(e1), pg, f"cuda:{dev}"))

    # ---- roofline of the dominant kernel (element Helmholtz, gather fused) ------
    prof = S.profile(iters=20)
    achieved = prof["op_bytes"] / (prof["op_ms"] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "helmholtz_hex_p%d_traffic.json" % (NM - 1))
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        traffic = tr["dram_bytes_per_element"] * P.mesh.nelmt
    it_ms = sum(prof[k] for k in ("op_ms", "assemble_ms", "update_ms", "scalars_ms"))
    it_bytes = prof["op_bytes"] + 8.0 * 11 * (nglob - ndir) + 8.0 * nloc + 4.0 * nloc + \
        20.0 * nglob
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic,
                "kernel": P.op.kernel(gather=True) + ": element Helmholtz, gather fused",
                "peak_source": peak_src, "kernel_ms": prof["op_ms"],
                "algorithmic_bytes": prof["op_bytes"], "algorithmic_flops": prof["op_flops"],
                "fp64_tflops": prof["op_flops"] / (prof["op_ms"] * 1e-3) / 1e12,
                "iteration_ms": {k: prof[k] for k in ("op_ms", "assemble_ms", "update_ms",
                                                      "scalars_ms")},
                "iteration": {"ms": it_ms, "algorithmic_bytes": it_bytes,
                              "frac": it_bytes / (it_ms * 1e-3) / 1e9 / hbm}}
    fp64_peak = max([v for v in (peaks_c.get("fp64_fma_tflops"), peaks_c.get("fp64_mma_tflops"))
                     if v] or [0.0])
    if fp64_peak:
        roofline["compute_frac"] = roofline["fp64_tflops"] / fp64_peak

    extras = {}
    rec = reference_iterations()
    if world == 1 and not args.no_extras:
        k2 = max(3, min(args.steps, 8))
        # ---- the converged FP64 solution, parity against the reference record --
        P.solve(TOL_CONVERGED)
        x_conv = P.x()
        parity = {"iterations": reps[-1].iterations,
                  "rms_error_vs_exact": P.rms_vs_exact(nb, x_fp64),
                  "rel_l2_vs_fp64_converged": _rel(x_fp64, x_conv)}
        dg = digest_check(rec, x_fp64, x_conv)
        if dg:
            parity.update(dg)
        extras["parity"] = parity
        extras["mixed"] = mixed_block(P, k2, x_conv, value)
        del x_conv
    P.close()

    if world == 1 and not args.no_extras:
        # ---- the P = 8 companion (24^3, Q = 10): FP64 and mixed --------------
        c3 = Problem(nb, torch, *WORKLOADS["hex24_p8"][:2], dev)
        c3.solve()
        ms3, reps3 = c3.timed(k2)
        x3 = c3.x()
        c3.solve(TOL_CONVERGED)
        x3c = c3.x()
        v3 = 1e3 * k2 / ms3
        c3rec = reference_record("c3")
        extras["c3"] = {"workload": WORKLOADS["hex24_p8"][2], "fp64": {
            "value": v3, "unit": "solves/s", "iterations": reps3[-1].iterations,
            "rel_l2_vs_fp64_converged": _rel(x3, x3c),
            "parity": digest_check(c3rec, x3, x3c)},
            "mixed": mixed_block(c3, k2, x3c, v3)}
        p3 = c3.S.profile(iters=10)
        extras["c3"]["fp64"]["operator_ms"] = p3["op_ms"]
        extras["c3"]["fp64"]["operator_frac"] = p3["op_bytes"] / (p3["op_ms"] * 1e-3) / 1e9 / hbm
        del x3, x3c
        c3.close()
        # ---- element operators alone at P = 4, 6, 8 (FP64 and FP32) ------------
        extras["operators"] = [operator_roofline(nb, torch, dev, n, p, prec, hbm, peaks=peaks_c)
                               for n, p in ((32, 4), (32, 6), (24, 8))
                               for prec in ("fp64", "fp32")]
        # ---- mixed-element batched apply (110000 hexes, prisms and tets) -------
        from nektar_b200 import mixedbench
        extras["c4"] = {prec: mixedbench.measure(precision=prec, iters=10, groups_detail=False,
                                                 device=dev)
                        for prec in ("fp64", "fp32")}

    its = [r.iterations for r in reps]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (manufactured solution, zero Dirichlet data)",
        "config": workload_config(P.mesh.nelmt, nloc, nglob, ndir, world),
        "iterations": its[-1], "rel_residual": reps[-1].rel_residual,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "helmholtz_gdof_s": nloc / (prof["op_ms"] * 1e-3) / 1e9,
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": 2 * nloc * 8,
                "d2h_bytes_per_step": nloc * 8},
        "roofline": roofline, "compute_peaks": peaks_c, "cpu_baseline": cpu_base,
        "clocks": clocks.summary(), "gpu_launches": int(sum(r.kernel_launches for r in reps)),
    }
    line.update(extras)
    replicas.finish(pg)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_shard(args, rank, world, local):
    """The headline solve sharded over the N GPUs: rank r holds elements
    partition(nelmt, N, r) and its dofs; per iteration the shared dofs go to
    the neighbour ranks by NCCL send/recv and the three dot sums through one
    NCCL all-reduce, inside the CUDA graph of the iterations (strong scaling:
    the whole job is one solve). Each step is one solve through the public
    call with host buffers (right-hand side in, solution out); `value` is
    timed by the device events around the solve (after the copy in, before
    the copy out), `e2e` by the wall clock around the call, both the maximum
    over ranks."""
    import time

    import torch
    import nektar_b200 as nb

    from nektar_b200 import replicas
    from nektar_b200.sharded import DeviceShardGroup, close_comm, make_comm, shard_plans
    torch.cuda.set_device(local)
    pg = replicas.init(world, local, "nccl")
    mesh = nb.BoxMesh("hex", N_CELLS, NM, NM + 1, amp=AMP, coords=True)
    gmap, nglob, ndir = mesh.assembly()
    nc, nt = mesh.nc, mesh.nt
    p = shard_plans(np.asarray(gmap), ndir, world, nc=nc)[rank]
    lo, hi = p["lo"], p["hi"]
    op = nb.Operator("helmholtz", shape="hex", nm=NM, nq=mesh.nq, nelmt=hi - lo, T=mesh.T,
                     jac=mesh.jac[lo * nt:hi * nt],
                     df=np.ascontiguousarray(mesh.df[:, lo * nt:hi * nt]), deformed=True,
                     device=local)
    op.set_factors(LAM)
    ipo = nb.Operator("iproduct", shape="hex", nm=NM, nq=mesh.nq, nelmt=hi - lo, T=mesh.T,
                      jac=mesh.jac[lo * nt:hi * nt], deformed=True, device=local)
    x, y, z = (c[lo * nt:hi * nt] for c in mesh.xyz)
    b = ipo((3 * np.pi ** 2 + LAM) * np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z))
    ipo.close()
    mesh.xyz = mesh.jac = mesh.df = None
    os.environ.setdefault("NCCL_DEBUG", "WARN")  # stdout carries the one JSON line
    comm = make_comm(pg, local)
    G = DeviceShardGroup([p], [[op]], comm=comm, device=local)
    b_pin = torch.tensor(b).pin_memory().numpy()
    for _ in range(max(args.warmup, 3)):
        G.solve([b_pin], tol=TOL, maxit=20000, check_interval=K_CHECK)
    dev_ms, wall, its = 0.0, 0.0, 0
    with ClockSampler(local) as clocks:
        replicas.barrier(pg)
        for _ in range(args.steps):
            t0 = time.perf_counter()
            _, reps = G.solve([b_pin], tol=TOL, maxit=20000, check_interval=K_CHECK)
            wall += time.perf_counter() - t0
            dev_ms += reps[0].device_ms
            its = reps[0].iterations
        replicas.barrier(pg)
    ms_max = replicas.max_over_ranks(dev_ms, pg, f"cuda:{local}")
    wall_max = replicas.max_over_ranks(wall, pg, f"cuda:{local}")
    nloc_r = (hi - lo) * nc
    G.close()
    close_comm(comm)
    op.close()
    line = {
        "metric": METRIC, "value": 1e3 * args.steps / ms_max, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (manufactured solution, zero Dirichlet data)",
        "config": dict(workload_config(mesh.nelmt, mesh.nelmt * nc, nglob, ndir, world),
                       parallelism="shard%d" % world),
        "iterations": its,
        "shard": {"elements_per_rank_max": int(-(-mesh.nelmt // world)),
                  "shared_dofs_rank0": int(p["shared"].size),
                  "neighbours_rank0": [int(q) for q in p["nbr"]]},
        "e2e": {"value": args.steps / wall_max, "unit": "solves/s",
                "h2d_bytes_per_step": 2 * nloc_r * 8, "d2h_bytes_per_step": nloc_r * 8},
        "clocks": clocks.summary(),
        "gpu_launches": int(reps[0].kernel_launches) * args.steps,
    }
    replicas.finish(pg)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.shard:
        run_shard(args, rank, world, local)
    else:
        run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
