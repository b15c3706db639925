"""Serving benchmark: a seeded stream of Helmholtz solve requests (Poisson
arrivals, curved hex boxes of log-uniform size and random order, random
lambda, half FP64 to 1e-10 and half mixed precision to 1e-8) served on one
GPU by the continuous-batching loop of nektar_b200.serve.

    python -m nektar_b200.servebench --requests 64 --rate 200 [--prewarm]

--prewarm builds every mesh context the stream needs before the clock
starts (meshes registered ahead of the requests; their setup is reported
separately); without it a request that brings a new mesh pays the setup
inside its latency. Prints one JSON line: solves/s, local DOF/s, latency
p50/p99, queueing, peak device bytes under the admission budget.
"""
import argparse
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--emin", type=int, default=1000)
    ap.add_argument("--emax", type=int, default=64000)
    ap.add_argument("--max-active", type=int, default=8)
    ap.add_argument("--budget-frac", type=float, default=0.8,
                    help="admission budget as a fraction of the free device memory")
    ap.add_argument("--prewarm", action="store_true")
    ap.add_argument("--detail", default=None,
                    help="write one JSON line per request (mesh, order, lambda, tolerance, "
                         "precision, iterations, convergence, times) to this file")
    a = ap.parse_args()
    import torch

    from nektar_b200.serve import CudaBackend, Scheduler, make_workload, summarize
    reqs = make_workload(a.requests, rate=a.rate, seed=a.seed, emin=a.emin, emax=a.emax)
    free, total = torch.cuda.mem_get_info()
    budget = int(a.budget_frac * free)
    be = CudaBackend()
    sch = Scheduler(be, budget, max_active=a.max_active)
    setup_s = 0.0
    if a.prewarm:
        t0 = time.perf_counter()
        sch.prewarm(list(dict.fromkeys(r.key for r in reqs)))
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = sch.run(reqs)
    wall = time.perf_counter() - t0
    s = summarize(res, reqs)
    s.update({
        "metric": "Helmholtz solve requests served per second (Poisson %g req/s)" % a.rate,
        "mode": "prewarmed contexts" if a.prewarm else "contexts built on demand",
        "prewarm_setup_s": setup_s, "wall_s": wall, "budget_bytes": budget,
        "peak_bytes": sch.peak, "max_active": a.max_active,
        "mixed_requests": sum(r.mixed for r in reqs),
        "distinct_meshes": len({r.key for r in reqs}),
        "iterations": {"p50": float(sorted(r.iterations for r in res)[len(res) // 2]),
                       "max": max(r.iterations for r in res)},
    })
    sch.close()
    if a.detail:
        by_id = {r.rid: r for r in reqs}
        with open(a.detail, "w") as f:
            for r in sorted(res, key=lambda r: r.rid):
                q = by_id[r.rid]
                f.write(json.dumps({"rid": r.rid, "n": q.n, "P": q.P, "lam": q.lam, "tol": q.tol,
                                    "mixed": q.mixed, "iterations": r.iterations,
                                    "converged": r.converged, "rel_residual": r.rel_residual,
                                    "device_ms": r.device_ms, "latency_s": r.latency,
                                    "new_context": r.new_context}) + "\n")
    print(json.dumps(s), flush=True)


if __name__ == "__main__":
    main()
