"""Serving loop for Helmholtz solves on one GPU.

Requests (a curved hex box of n^3 elements at order P, a Helmholtz lambda, a
tolerance, FP64 or mixed precision, a right-hand side) arrive over time. The
server keeps everything device resident and runs many solves at once:

* a *context* per mesh (n, P) holds what solves of that mesh share: the FP64
  and FP32 element operators (packed geometry), the local->global map with its
  CSR inverse and the split Jacobi diagonal (nkb_sys_create);
* a *slot* is one solve in flight on a context: a clone of the context's
  system (nkb_sys_clone: own CG vectors, own lambda via nkb_sys_set_lambda),
  its own CUDA stream, device buffers for b and x and pinned host buffers;
  finished slots go back to their context for reuse;
* admission is by HBM footprint: a request is admitted (FIFO) when its
  context (if not resident) and a slot fit in the byte budget; idle contexts
  are evicted least-recently-used to make room;
* continuous batching: every active solve is advanced with the non-blocking
  nkb_cg_poll, one block of check_interval iterations at a time, so new
  requests join while others are mid-solve and small solves fill the GPU
  next to large ones.

The scheduler (`Scheduler`) only sees the `Backend` interface, so its policy
is testable on the CPU with a fake backend; `CudaBackend` is the device one.
A solve's result does not depend on what else is in flight: each slot's
kernels, reductions and stopping decisions are its own (the tests check
bitwise equality with the same request served alone).
"""
import collections
import dataclasses
import math
import time

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float      # seconds after the start of the run
    n: int              # n^3 hex elements
    P: int              # polynomial order (nm = P + 1, Q = P + 2)
    lam: float          # Helmholtz lambda
    tol: float          # relative residual tolerance
    mixed: bool         # FP32 CG with FP64 reliable updates
    seed: int           # right-hand side: uniform(-1, 1) local coefficients

    @property
    def key(self):
        return (self.n, self.P)


@dataclasses.dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    rel_residual: float
    device_ms: float
    new_context: bool
    x: object = None    # local solution (host array) when kept

    @property
    def latency(self):
        return self.finished - self.arrival


def make_workload(num, rate=200.0, seed=0, emin=1000, emax=64000, pmin=3, pmax=8,
                  lam_range=(0.1, 10.0)):
    """Seeded synthetic request stream: Poisson arrivals at `rate` per second,
    element count log-uniform in [emin, emax] rounded to the nearest cube
    n^3, P uniform in {pmin..pmax}, lambda uniform in lam_range, and with
    probability 1/2 a mixed-precision solve to 1e-8, else FP64 to 1e-10."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, num))
    e = np.exp(rng.uniform(math.log(emin), math.log(emax), num))
    n = np.maximum(1, np.rint(np.cbrt(e))).astype(int)
    P = rng.integers(pmin, pmax + 1, num)
    lam = rng.uniform(lam_range[0], lam_range[1], num)
    mixed = rng.random(num) < 0.5
    seeds = rng.integers(0, 2 ** 31 - 1, num)
    return [Request(i, float(t[i]), int(n[i]), int(P[i]), float(lam[i]),
                    1e-8 if mixed[i] else 1e-10, bool(mixed[i]), int(seeds[i]))
            for i in range(num)]


def rhs_for(req, nloc):
    return np.random.default_rng(req.seed).uniform(-1.0, 1.0, nloc)


# ---------------------------------------------------------------------------
# scheduler
# ---------------------------------------------------------------------------

class Scheduler:
    """FIFO admission by device-memory footprint, LRU eviction of idle
    contexts, continuous batching of the admitted solves through
    non-blocking polls."""

    def __init__(self, backend, budget_bytes, max_active=8, keep_x=False, clock=None,
                 idle_sleep=2e-4):
        self.backend = backend
        self.budget = int(budget_bytes)
        self.max_active = max_active
        self.keep_x = keep_x
        self.clock = clock or time.perf_counter
        self.idle_sleep = idle_sleep
        self.contexts = collections.OrderedDict()   # key -> context (LRU order)
        self.used = 0
        self.peak = 0

    # -- memory ------------------------------------------------------------
    def _charge(self, nbytes):
        self.used += nbytes
        self.peak = max(self.peak, self.used)

    def _evict_for(self, need, keep_key):
        """Free idle contexts (no active slot), least recently used first,
        until `need` more bytes fit. Returns True when they fit."""
        for key in list(self.contexts):
            if self.used + need <= self.budget:
                break
            ctx = self.contexts[key]
            if key == keep_key or ctx.active:
                continue
            self.used -= ctx.total_bytes()
            ctx.close()
            del self.contexts[key]
        return self.used + need <= self.budget

    def _try_admit(self, req):
        """Context + slot for `req`, or None when they do not fit now."""
        ctx = self.contexts.get(req.key)
        new_ctx = ctx is None
        need = 0
        if new_ctx:
            need += self.backend.context_bytes(req.key)
        slot_fresh = new_ctx or not ctx.idle
        if slot_fresh:
            need += self.backend.slot_bytes(req.key)
        if need > self.budget:
            raise MemoryError("request %d needs %d bytes, more than the budget %d"
                              % (req.rid, need, self.budget))
        if self.used + need > self.budget and not self._evict_for(need, req.key):
            return None
        if new_ctx:
            ctx = self.backend.create_context(req.key)
            self.contexts[req.key] = ctx
            self._charge(ctx.bytes)
        self.contexts.move_to_end(req.key)
        if ctx.idle:
            slot = ctx.idle.pop()
        else:
            slot = ctx.new_slot()
            self._charge(slot.bytes)
        ctx.active += 1
        return ctx, slot, new_ctx

    def prewarm(self, keys):
        """Build the contexts (and one slot each) for `keys` before any
        request arrives, while they fit in the budget; returns the keys
        built."""
        built = []
        for key in keys:
            got = self._try_admit(Request(-1, 0.0, key[0], key[1], 1.0, 1e-10, False, 0))
            if got is None:
                break
            ctx, slot, _ = got
            ctx.active -= 1
            ctx.idle.append(slot)
            built.append(key)
        return built

    # -- run ---------------------------------------------------------------
    def run(self, requests):
        """Serve `requests` (sorted by arrival) in real time; returns the
        results in request order."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue = collections.deque()
        active = []
        results = {}
        t0 = self.clock()
        while pending or queue or active:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            progressed = False
            while queue and len(active) < self.max_active:
                got = self._try_admit(queue[0])
                if got is None:
                    break
                req = queue.popleft()
                ctx, slot, new_ctx = got
                slot.start(req)
                active.append((req, ctx, slot, new_ctx, self.clock() - t0))
                progressed = True
            still = []
            for item in active:
                req, ctx, slot, new_ctx, t_adm = item
                if slot.advance():
                    rep, x = slot.finish()
                    results[req.rid] = Result(
                        req.rid, req.arrival, t_adm, self.clock() - t0, rep["iterations"],
                        rep["converged"], rep["rel_residual"], rep["device_ms"], new_ctx,
                        x if self.keep_x else None)
                    ctx.active -= 1
                    ctx.idle.append(slot)
                    progressed = True
                else:
                    still.append(item)
            active = still
            if not progressed:
                if not active and not queue and pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (self.clock() - t0), 0.01)))
                else:
                    time.sleep(self.idle_sleep)
        return [results[r.rid] for r in requests]

    def close(self):
        for ctx in self.contexts.values():
            ctx.close()
        self.contexts.clear()
        self.used = 0


def summarize(results, requests, wall_s=None):
    lat = np.array([r.latency for r in results])
    t_first = min(r.arrival for r in results)
    t_last = max(r.finished for r in results)
    span = wall_s if wall_s is not None else t_last - t_first
    dofs = sum(req.n ** 3 * (req.P + 1) ** 3 for req in requests)
    return {
        "requests": len(results),
        "solves_per_s": len(results) / span,
        "local_dofs_per_s": dofs / span,
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "mean": float(lat.mean()), "max": float(lat.max())},
        "queue_s": {"p50": float(np.percentile([r.admitted - r.arrival for r in results], 50)),
                    "p99": float(np.percentile([r.admitted - r.arrival for r in results], 99))},
        "converged": int(sum(r.converged for r in results)),
        "new_contexts": int(sum(r.new_context for r in results)),
        "span_s": span,
    }


# ---------------------------------------------------------------------------
# device backend
# ---------------------------------------------------------------------------

def _op_bytes(nelmt, nm, nq, fp32):
    """Device bytes of one Helmholtz operator on nelmt hexes: raw J and the 9
    derivative factors per point (kept for factor updates), the packed FP64
    geometry (7 values per point, element stride rounded to 4) and, for an
    FP32 operator, its FP32 copy."""
    nt = nq ** 3
    gstride = (7 * nt + 3) & ~3
    b = nelmt * nt * 10 * 8 + nelmt * gstride * 8
    if fp32:
        b += nelmt * gstride * 4
    return b + 64 * 1024


class CudaSlot:
    """One solve in flight: a clone of the context's system with its own
    lambda and stream, device b / x and pinned host b / x."""

    def __init__(self, ctx):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.sys = ctx.sys.clone()
        nloc = ctx.sys.nloc
        dev = ctx.device
        self.stream = torch.cuda.Stream(device=dev)
        self.b = torch.empty(nloc, dtype=torch.float64, device="cuda:%d" % dev)
        self.x = torch.empty(nloc, dtype=torch.float64, device="cuda:%d" % dev)
        self.hb = torch.empty(nloc, dtype=torch.float64).pin_memory()
        self.hx = torch.empty(nloc, dtype=torch.float64).pin_memory()
        self.done_ev = torch.cuda.Event()
        self.bytes = self.sys.footprint()[1] + 2 * nloc * 8
        self.phase = 0
        self.rep = None

    def start(self, req):
        torch = self.torch
        self.req = req
        self.hb.numpy()[:] = rhs_for(req, self.ctx.sys.nloc)
        self.sys.set_lambda(req.lam)
        with torch.cuda.stream(self.stream):
            self.b.copy_(self.hb, non_blocking=True)
            self.x.zero_()
        self.sys.begin(self.b.data_ptr(), self.x.data_ptr(), tol=req.tol,
                       check_interval=self.ctx.check_interval, mixed=req.mixed,
                       stream=self.stream.cuda_stream, maxit=20000)
        self.phase = 1

    def advance(self):
        """True once the solution is back in host memory."""
        if self.phase == 1:
            if not self.sys.poll():
                return False
            self.rep = self.sys.end(raise_on_maxit=False)
            with self.torch.cuda.stream(self.stream):
                self.hx.copy_(self.x, non_blocking=True)
                self.done_ev.record(self.stream)
            self.phase = 2
        if self.phase == 2:
            if not self.done_ev.query():
                return False
            self.phase = 0
            return True
        return False

    def finish(self):
        r = self.rep
        rep = {"iterations": r.iterations, "converged": bool(r.converged),
               "rel_residual": r.rel_residual, "device_ms": r.device_ms}
        return rep, self.hx.numpy().copy()

    def close(self):
        self.sys.close()


class CudaContext:
    """Everything the solves of one mesh share."""

    def __init__(self, key, device, check_interval):
        import nektar_b200 as nb
        n, P = key
        nm = P + 1
        self.key, self.device, self.check_interval = key, device, check_interval
        # the geometric factors are computed on the device and copied there
        # into both operators
        m = nb.BoxMesh("hex", n, nm, nm + 1, amp=0.05, geom_device=device)
        self.mesh = m
        gmap, nglob, ndir = m.assembly()
        jac, df = m.jac, m.df
        m.jac = m.df = None
        kw = dict(shape="hex", nm=nm, nq=m.nq, nelmt=m.nelmt, T=m.T, jac=jac, df=df,
                  deformed=m.deformed, device=device)
        self.op = nb.Operator("helmholtz", **kw)
        self.op32 = nb.Operator("helmholtz", precision="fp32", **kw)
        del jac, df, kw
        self.sys = nb.GlobalLinSys([self.op], gmap, nglob, ndir, device=device, ops32=[self.op32])
        shared, inst = self.sys.footprint()
        self.bytes = (_op_bytes(self.mesh.nelmt, nm, nm + 1, False)
                      + _op_bytes(self.mesh.nelmt, nm, nm + 1, True) + shared + inst)
        self.idle = []
        self.slots = []
        self.active = 0

    def new_slot(self):
        s = CudaSlot(self)
        self.slots.append(s)
        return s

    def total_bytes(self):
        return self.bytes + sum(s.bytes for s in self.slots)

    def close(self):
        for s in self.slots:
            s.close()
        self.slots, self.idle = [], []
        self.sys.close()
        self.op.close()
        self.op32.close()


class CudaBackend:
    def __init__(self, device=0, check_interval=16):
        self.device = device
        self.check_interval = check_interval

    @staticmethod
    def _sizes(key):
        n, P = key
        nm = P + 1
        nelmt = n ** 3
        nloc = nelmt * nm ** 3
        nglob = (n * P + 1) ** 3
        return nelmt, nm, nloc, nglob

    def context_bytes(self, key):
        nelmt, nm, nloc, nglob = self._sizes(key)
        ops = _op_bytes(nelmt, nm, nm + 1, False) + _op_bytes(nelmt, nm, nm + 1, True)
        shared = nloc * 8 + (nglob + 1) * 4 + 2 * nglob * 8
        return ops + shared + self.slot_bytes(key)

    def slot_bytes(self, key):
        nelmt, nm, nloc, nglob = self._sizes(key)
        fp64 = (4 * nglob + 4 * nglob) * 8 + 2 * nloc * 8
        fp32 = (4 * nglob + 4 * nglob) * 4 + nloc * 4
        return fp64 + fp32 + 2 * nloc * 8 + 1024 * 1024

    def create_context(self, key):
        return CudaContext(key, self.device, self.check_interval)
