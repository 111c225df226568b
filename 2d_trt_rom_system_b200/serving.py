"""Request loop for many independent solves on one GPU: admission against an HBM budget and continuous
batching.

Each request is an independent time-dependent solve (its own grid, groups, quadrature and materials)
that runs the transport-only time loop on its own resident handle (own CUDA stream).  A dispatcher
admits queued requests in arrival order whenever the device memory they need fits in what the budget
has left; admitted requests run concurrently, one host thread each (the library's calls release the
interpreter lock while they wait on their stream), so their kernels overlap on the device.  A request
that arrives while others run is admitted as soon as memory frees up.  Per-step and per-solve
latencies are recorded for p50/p99 reporting.

Results do not depend on what else runs: every kernel of a handle reads and writes only that handle's
memory and every reduction has a fixed order, so a solve is bit-identical alone and in a mix.
"""
import dataclasses
import math
import threading
import time

import numpy as np

from . import problems as P


@dataclasses.dataclass
class Request:
    rid: int
    arrival_s: float                # arrival time after the stream starts
    prob: P.Problem
    steps: int = 10
    precision: str = "mixed"
    maxit: int = 4                  # outer iterations per time step (conv_ho below is rarely met first)
    conv_ho: float = 1e-8


@dataclasses.dataclass
class Result:
    rid: int
    arrival_s: float
    admitted_s: float
    finished_s: float
    bytes: int
    updates: int                    # cell-direction-group updates swept
    step_ms: list
    its: list
    T: np.ndarray = None
    error: str = ""

    @property
    def solve_s(self):
        return self.finished_s - self.arrival_s


def config3_requests(rate=200.0, duration=60.0, seed=3, steps=10, precision="mixed", maxit=4):
    """Poisson arrivals at `rate` per second for `duration` seconds (seed 3): grid N log-uniform in
    [32, 384], 17-64 groups, S8 or S16, random materials as in config 2."""
    rng = np.random.default_rng(seed)
    out, t, k = [], 0.0, 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            return out
        n = int(round(math.exp(rng.uniform(math.log(32), math.log(384)))))
        G = int(rng.integers(17, 65))
        quad = "S8" if rng.uniform() < 0.5 else "S16"
        kappa0, cv = P._paint_rectangles(rng, n, n, 6.0, 6.0, 6, lambda r: float(10 ** r.uniform(0.0, 4.0)),
                                         lambda r: float(r.uniform(0.1, 1.0)))
        tbc = float(rng.uniform(0.5, 2.0))
        prob = P.Problem(f"C3-{k}", n, n, 6.0, 6.0, P.log_groups(G), quad, kappa0, cv, 0.01, (tbc, 0.0, 0.0, 0.0),
                         steps=steps)
        out.append(Request(k, t, prob, steps=steps, precision=precision, maxit=maxit))
        k += 1


def config2_batch(count=64, steps=10, precision="mixed", maxit=4):
    """Config 2: `count` independent instances (seed 2), all present at t = 0."""
    return [Request(k, 0.0, p, steps=steps, precision=precision, maxit=maxit)
            for k, p in enumerate(P.config2_instances(count))]


def required_bytes(req):
    """Device bytes a request's handle may allocate (the library's estimate plus the time-loop fields)."""
    from . import api
    p = req.prob
    b = api.required_bytes(p.nx, p.ny, p.nm, p.ng, req.precision)
    return int(b + 10 * p.nx * p.ny * 8 + 4 * 1024 * 1024)


def _setup(s, req):
    """Initial state and the time loop of a request on handle s: the request's own material (the
    configurations' opacity law on its rectangles, c_v per cell), its boundary and initial temperature."""
    p = req.prob
    ts = P.config_timestep_setup(p)
    s.init_state(ts.Tini_eV, list(ts.bcT_eV), P.COMP_UNIT, ts.nu_eV)
    s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((p.nx, p.ny), ts.Tini_eV), ts.Kap0, P.COMP_UNIT,
                  P.C_LIGHT, ts.dt, bcT=ts.bcT_eV, conv_type=2, conv_ho=req.conv_ho, maxit_rte=req.maxit, law=1)


def solve(req, t0):
    """Run one request on its own handle, capped at its reserved bytes; returns a Result (times
    relative to t0)."""
    from . import api
    p = req.prob
    res = Result(req.rid, req.arrival_s, time.perf_counter() - t0, 0.0, required_bytes(req), 0, [], [])
    ox, oy, w = p.directions()
    try:
        with api.TransportSweep(p.nx, p.ny, ox, oy, w, p.delx, p.dely, p.ng, precision=req.precision,
                                hbm_budget=res.bytes) as s:
            _setup(s, req)
            for _ in range(req.steps):
                a = time.perf_counter()
                its, _, _ = s.tstep()
                res.step_ms.append((time.perf_counter() - a) * 1e3)
                res.its.append(its)
            res.T = s.temperature()
    except Exception as e:   # reported per request; the server keeps running
        res.error = f"{type(e).__name__}: {e}"
    res.updates = int(p.updates_per_sweep() * sum(res.its))
    res.finished_s = time.perf_counter() - t0
    return res


class Server:
    """Admits requests in arrival order against `hbm_budget` bytes (and at most `max_active` at once)
    and runs each admitted request on its own thread and handle."""

    def __init__(self, hbm_budget, max_active=64, solver=solve, sizer=required_bytes):
        self.budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.solver = solver
        self.sizer = sizer

    def run(self, requests, realtime=True):
        """Serve `requests`.  With realtime, a request is not admitted before its arrival time on the
        wall clock.  Returns the Results in request order and the admission log
        [(time, rid, bytes in use after admission)]."""
        reqs = sorted(requests, key=lambda r: (r.arrival_s, r.rid))
        sizes = {r.rid: self.sizer(r) for r in reqs}
        for r in reqs:
            if sizes[r.rid] > self.budget:
                raise ValueError(f"request {r.rid} needs {sizes[r.rid]} bytes, more than the budget {self.budget}")
        cv = threading.Condition()
        in_use = [0]
        active = [0]
        results = {}
        log = []
        t0 = time.perf_counter()

        def worker(r):
            res = self.solver(r, t0)
            with cv:
                in_use[0] -= sizes[r.rid]
                active[0] -= 1
                results[r.rid] = res
                cv.notify_all()

        threads = []
        queue = []
        nxt = 0
        with cv:
            while len(results) < len(reqs):
                now = time.perf_counter() - t0
                while nxt < len(reqs) and (not realtime or reqs[nxt].arrival_s <= now):
                    queue.append(reqs[nxt])
                    nxt += 1
                # admit in arrival order while the head of the queue fits
                while queue and active[0] < self.max_active and in_use[0] + sizes[queue[0].rid] <= self.budget:
                    r = queue.pop(0)
                    in_use[0] += sizes[r.rid]
                    active[0] += 1
                    log.append((time.perf_counter() - t0, r.rid, in_use[0]))
                    th = threading.Thread(target=worker, args=(r,), daemon=True)
                    th.start()
                    threads.append(th)
                if len(results) == len(reqs):
                    break
                wait = 1.0
                if nxt < len(reqs) and realtime:
                    wait = max(0.0, reqs[nxt].arrival_s - (time.perf_counter() - t0))
                cv.wait(timeout=wait)
        for th in threads:
            th.join()
        return [results[r.rid] for r in requests], log


class BatchedServer:
    """Continuous batching at time-step granularity: one driver steps every admitted solve together with
    trt_batch_tstep (one sweep launch per tiling class over all their CTAs); between steps, finished
    solves leave (their memory returns to the budget) and queued ones that now fit join, in arrival
    order.  Every member of a batched step sees that step's wall time as its per-step latency."""

    def __init__(self, hbm_budget, max_active=256, sizer=required_bytes):
        self.budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.sizer = sizer

    @staticmethod
    def _open(req):
        from . import api
        p = req.prob
        ox, oy, w = p.directions()
        s = api.TransportSweep(p.nx, p.ny, ox, oy, w, p.delx, p.dely, p.ng, precision=req.precision,
                               hbm_budget=required_bytes(req))
        try:
            _setup(s, req)
        except Exception:
            s.close()
            raise
        return s

    def run(self, requests, realtime=True):
        from . import api
        reqs = sorted(requests, key=lambda r: (r.arrival_s, r.rid))
        sizes = {r.rid: self.sizer(r) for r in reqs}
        for r in reqs:
            if sizes[r.rid] > self.budget:
                raise ValueError(f"request {r.rid} needs {sizes[r.rid]} bytes, more than the budget {self.budget}")
        t0 = time.perf_counter()
        self.stepping_s = 0.0                          # wall time spent in batched steps
        self.stepped_updates = 0
        results, log, queue, active = {}, [], [], []   # active: [request, handle, Result]
        in_use, nxt = 0, 0
        while len(results) < len(reqs):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival_s <= now):
                queue.append(reqs[nxt])
                nxt += 1
            while queue and len(active) < self.max_active and in_use + sizes[queue[0].rid] <= self.budget:
                r = queue.pop(0)
                res = Result(r.rid, r.arrival_s, time.perf_counter() - t0, 0.0, sizes[r.rid], 0, [], [])
                try:
                    h = self._open(r)
                except Exception as e:
                    res.error = f"{type(e).__name__}: {e}"
                    res.finished_s = time.perf_counter() - t0
                    results[r.rid] = res
                    continue
                in_use += sizes[r.rid]
                active.append([r, h, res])
                log.append((time.perf_counter() - t0, r.rid, in_use))
            if not active:
                if nxt < len(reqs):
                    time.sleep(max(0.0, reqs[nxt].arrival_s - (time.perf_counter() - t0)))
                continue
            a = time.perf_counter()
            try:
                with api.Batch([m[1] for m in active]) as b:
                    its, _, _ = b.tstep()
                err = ""
            except Exception as e:   # the whole step failed: report it on every member
                its, err = [0] * len(active), f"{type(e).__name__}: {e}"
            ms = (time.perf_counter() - a) * 1e3
            self.stepping_s += ms * 1e-3
            self.stepped_updates += sum(int(m[0].prob.updates_per_sweep()) * int(n) for m, n in zip(active, its))
            keep = []
            for (r, h, res), n_it in zip(active, its):
                res.step_ms.append(ms)
                res.its.append(int(n_it))
                if err:
                    res.error = err
                if err or len(res.its) == r.steps:
                    if not err:
                        res.T = h.temperature()
                    h.close()
                    in_use -= sizes[r.rid]
                    res.updates = int(r.prob.updates_per_sweep() * sum(res.its))
                    res.finished_s = time.perf_counter() - t0
                    results[r.rid] = res
                else:
                    keep.append([r, h, res])
            active = keep
        return [results[r.rid] for r in requests], log


def latency_summary(results):
    """p50/p99 per-step and per-solve latency, throughput and counts of a served stream."""
    ok = [r for r in results if not r.error]
    steps = np.array([x for r in ok for x in r.step_ms]) if ok else np.zeros(1)
    solves = np.array([r.solve_s * 1e3 for r in ok]) if ok else np.zeros(1)
    span = (max(r.finished_s for r in ok) - min(r.arrival_s for r in ok)) if ok else 1.0
    return {"requests": len(results), "failed": len(results) - len(ok),
            "errors": sorted({r.error for r in results if r.error})[:3],
            "step_ms_p50": float(np.percentile(steps, 50)), "step_ms_p99": float(np.percentile(steps, 99)),
            "solve_ms_p50": float(np.percentile(solves, 50)), "solve_ms_p99": float(np.percentile(solves, 99)),
            "updates_per_s": float(sum(r.updates for r in ok) / span), "span_s": float(span)}
