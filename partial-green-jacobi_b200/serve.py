"""Continuous-batching server for certified homogenizations and topology-optimization design steps.

One host loop drives one GPU. Work arrives as

* ``Homogenize``: one density multiplier field and a preconditioner exponent alpha; the result is
  the certified 6-load C_H.
* ``Lineage``: a design being optimised for ``steps`` design steps (the Study II outer loop of
  ``exp/asg_sctop_reproduction_20261105/reproduction.py:121-176``). Each step filters and projects
  the design (cone filter of radius ``rmin``, tanh projection, SIMP), runs a certified 6-load
  homogenization warm-started from the lineage's previous displacements, forms the shear
  objective and its sensitivity from the per-element energies, and applies the damped OC update
  with move limit ``move``. Filter, projection, solve, energies and OC all run on the device;
  the lineage's design fields and its six displacement fields stay resident between steps.

Admission is by an HBM budget: a request starts when a worker (a libpgj context of its grid size
with its own CUDA stream) is free, or a new one fits the budget, and when the lineage's resident
state fits. Requests that arrive while others are on the GPU are admitted as workers and memory
free up, so their work overlaps on the device (continuous batching, not a queue in front of one
solver). Every step is issued asynchronously; the loop polls CUDA events and never waits for one
request while others could be admitted. Results are identical whether a request runs alone or in a
mix: each context is private to one request at a time and every kernel reduces in a fixed order.

Precision. A mixed server runs FP32 inner recurrences (FP64 certificate); any mixed request that
fails certification is redone in FP64, warm-started from the mixed iterate, and lineages whose Emin is
below ``fp64_below_emin`` (default 0: none) run in FP64 from the start. A lineage without a fixed alpha
takes the eta-lookup exponent of its weak-material ratio (9/16, 11/16, 13/16 for Emin 1e-4, 1e-6,
1e-9; the reference's replay study, exp/asg_density_selector_20261105/run.py:57), with which the
mixed recurrence certifies up to Emin 1e-9. A design step commits its OC update only once its solve
is certified.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from . import _lib
from .designs import baseline_density
from .outer import PaperOuter
from .resident import ETA_ANCHORS, PAPER_MEDIUM, Operator


def _torch():
    import torch

    return torch


def eta_alpha(emin: float) -> float:
    """Eta-lookup exponent of the nearest calibrated weak-material ratio (log scale)."""
    return ETA_ANCHORS[min(ETA_ANCHORS, key=lambda k: abs(math.log10(k) - math.log10(emin)))]


def supported_n(n: int) -> bool:
    """Grid edges libpgj accepts: even, 4 <= n <= 256, FFT radices 2, 3, 5."""
    if n < 4 or n > 256 or n % 2:
        return False
    m = n
    for r in (2, 3, 5):
        while m % r == 0:
            m //= r
    return m == 1


def snap_n(n: float) -> int:
    """Nearest supported grid edge (ties to the smaller)."""
    best = None
    for m in range(4, 257, 2):
        if supported_n(m) and (best is None or abs(m - n) < abs(best - n)):
            best = m
    return best


@dataclass
class Homogenize:
    a: object            # (n, n, n) density multiplier (host or device)
    alpha: float = 0.5
    tag: object = None


@dataclass
class Lineage:
    n: int
    seed: int
    emin: float = 1e-6
    steps: int = 30
    volume: float = 0.3
    alpha: float | None = None  # None: the eta lookup of emin
    rmin: float = 1.5
    move: float = 0.2
    beta: float = 4.0
    eta: float = 0.5
    tag: object = None


@dataclass
class Arrival:
    t: float             # seconds after the start of the run
    req: object          # Homogenize | Lineage


@dataclass
class StepResult:
    tag: object
    kind: str            # "homogenize" | "design_step"
    step: int
    n: int
    C: np.ndarray
    objective: float
    status: int
    iterations: int      # most PCG iterations over the six loads
    queued_ms: float     # ready -> admitted (host clock)
    latency_ms: float    # ready -> result on the host (host clock)
    device_ms: float     # first to last device operation of the step (CUDA events)
    oc_steps: int = 0
    change: float = 0.0
    precision: str = ""  # "mixed", "fp64", or "fp64-fallback" (redone after a mixed failure)


class _Worker:
    def __init__(self, n: int, precision: str, lam: float, mu: float):
        torch = _torch()
        self.n = n
        self.precision = precision
        self.stream = torch.cuda.Stream()
        with torch.cuda.stream(self.stream):
            self.op = Operator(n, 6, lam, mu, precision)
            self.u0 = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
            self.Cd = torch.empty((6, 6), dtype=torch.float64, device="cuda")
            self.scal = torch.zeros(4, dtype=torch.float64, device="cuda")
        self.Ch = torch.empty((6, 6), dtype=torch.float64).pin_memory()
        self.sh = torch.empty(4, dtype=torch.float64).pin_memory()
        self.bytes = worker_bytes(n, precision)
        self.job = None
        self.last_used = 0.0


class _LineageState:
    def __init__(self, spec: Lineage):
        torch = _torch()
        self.spec = spec
        n = spec.n
        self.outer = PaperOuter(n, spec.volume, spec.rmin, spec.beta, spec.eta, spec.emin, spec.move)
        self.outer.set_initial(baseline_density(n, spec.seed, spec.volume))
        self.u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")  # warm start
        self.step = 0
        self.bytes = lineage_bytes(n)
        self.pending_advance = False  # the last certified step's OC update waits to be committed


@dataclass
class _Job:
    req: object
    ready: float                     # host time the request became ready (arrival or previous step)
    lineage: _LineageState | None = None
    step: int = 0
    admitted: float = 0.0
    start: object = None
    end: object = None
    precision: str = "fp64"
    fallback: bool = False           # FP64 redo of a mixed request that failed certification
    u_start: object = None           # homogenization redo: the mixed iterate as the FP64 warm start


def worker_bytes(n: int, precision: str) -> int:
    import ctypes as C

    nb = C.c_size_t()
    _lib.check(_lib.lib().pgj_workspace_bytes(n, 6, _lib.PGJ_FP32 if precision == "mixed" else _lib.PGJ_FP64,
                                              C.byref(nb)), "pgj_workspace_bytes")
    return int(nb.value) + 256 + 8 * 18 * n ** 3 + 4096


def lineage_bytes(n: int) -> int:
    N = n ** 3
    # PaperOuter fields (8 N) and OC scratch (4 N + 512), warm-start displacements (18 N), energies (6 N)
    return 8 * (8 * N + 4 * N + 512 + 18 * N + 6 * N)


class Server:
    """Continuous batching over libpgj contexts under an HBM budget (bytes)."""

    def __init__(self, precision: str = "mixed", hbm_budget: float = 120e9, max_workers_per_n: int = 4,
                 rtol: float = 1e-8, medium=PAPER_MEDIUM, fp64_below_emin: float = 0.0, fallback: bool = True):
        self.precision = precision
        self.fp64_below_emin = float(fp64_below_emin)
        self.fallback = bool(fallback)
        self.fallbacks = 0     # mixed requests redone in FP64
        self.budget = int(hbm_budget)
        self.max_workers_per_n = int(max_workers_per_n)
        self.rtol = float(rtol)
        self.lam, self.mu = medium
        self.macros = np.ascontiguousarray(np.eye(6))
        self.workers: list[_Worker] = []
        self.used = 0          # bytes held by workers and resident lineages
        self.peak_used = 0
        self.max_inflight = 0  # most requests on the device at once

    def warm(self, requests) -> None:
        """Create one worker (context, stream, solve graph) for every grid size and precision these
        requests will use, outside any timed run."""
        torch = _torch()
        kinds = sorted({(self._n_of(r), self._precision_for(r)) for r in requests}
                       | ({(self._n_of(r), "fp64") for r in requests} if self.precision == "mixed" else set()))
        for n, prec in kinds:
            w = self._worker_for(n, prec, 0)
            if w is None:
                continue
            with torch.cuda.stream(w.stream):
                a = torch.ones((n, n, n), dtype=torch.float64, device="cuda")
                w.op.set_material(a)
                w.op.set_alpha(0.5)
                w.u0.zero_()
                w.op.solve(self.macros, self.rtol, w.u0)  # homogeneous: certifies at once, builds the graphs
        torch.cuda.synchronize()

    # ----------------------------------------------------------------------------- admission
    def _n_of(self, req) -> int:
        return int(req.n) if isinstance(req, Lineage) else int(req.a.shape[0])

    def _need(self, job: _Job) -> int:
        return lineage_bytes(job.req.n) if isinstance(job.req, Lineage) and job.lineage is None else 0

    def _precision_for(self, req) -> str:
        if self.precision == "mixed" and isinstance(req, Lineage) and req.emin < self.fp64_below_emin:
            return "fp64"
        return self.precision

    def _worker_for(self, n: int, prec: str, extra: int) -> _Worker | None:
        free = [w for w in self.workers if w.n == n and w.precision == prec and w.job is None]
        if free:
            return free[0] if self.used + extra <= self.budget else None
        if sum(1 for w in self.workers if w.n == n and w.precision == prec) >= self.max_workers_per_n:
            return None
        need = worker_bytes(n, prec) + extra
        # evict idle workers of other kinds, least recently used first, while over budget
        idle = sorted((w for w in self.workers if w.job is None and (w.n != n or w.precision != prec)),
                      key=lambda w: w.last_used)
        while self.used + need > self.budget and idle:
            w = idle.pop(0)
            self.workers.remove(w)
            self.used -= w.bytes
        if self.used + need > self.budget:
            return None
        w = self._new_worker(n, prec)
        self.workers.append(w)
        self.used += w.bytes
        return w

    def _new_worker(self, n: int, prec: str) -> _Worker:
        return _Worker(n, prec, self.lam, self.mu)

    def _snapshot_iterate(self, w: _Worker):
        """Copy of a worker's homogenization iterate, complete before the call returns."""
        u = w.u0.clone()
        _torch().cuda.current_stream().synchronize()
        return u

    def _drain(self) -> None:
        _torch().cuda.synchronize()

    # ----------------------------------------------------------------------------- launch / finish
    def _launch(self, w: _Worker, job: _Job) -> None:
        torch = _torch()
        L = _lib.lib()
        w.job = job
        job.admitted = time.perf_counter()
        with torch.cuda.stream(w.stream):
            job.start = torch.cuda.Event(enable_timing=True)
            job.start.record(w.stream)
            if isinstance(job.req, Lineage):
                if job.lineage is None:
                    job.lineage = _LineageState(job.req)
                    self.used += job.lineage.bytes
                ls = job.lineage
                if ls.pending_advance:                  # commit the previous certified step's update
                    ls.outer.advance()
                    ls.pending_advance = False
                ls.outer.evaluate()                     # filter + projection + SIMP -> outer.a
                w.op.set_material(ls.outer.a)
                w.op.set_alpha(job.req.alpha if job.req.alpha is not None else eta_alpha(job.req.emin))
                u = ls.u                                # warm start, updated in place
            else:
                a = torch.as_tensor(job.req.a, dtype=torch.float64)
                a = a.to("cuda", non_blocking=True) if not a.is_cuda else a
                w.op.set_material(a.contiguous())
                w.op.set_alpha(job.req.alpha)
                if job.u_start is not None:
                    w.u0.copy_(job.u_start)             # the mixed iterate
                else:
                    w.u0.zero_()
                u = w.u0
            _lib.check(L.pgj_solve_async(w.op._ctx, 6, self.macros.ctypes.data, self.rtol, u.data_ptr(),
                                         w.stream.cuda_stream), "pgj_solve_async")
            _lib.check(L.pgj_effective_tensor(w.op._ctx, u.data_ptr(), w.Cd.data_ptr(), w.stream.cuda_stream),
                       "pgj_effective_tensor")
            w.Ch.copy_(w.Cd, non_blocking=True)
            if isinstance(job.req, Lineage):
                ls = job.lineage
                e = w.op.energies(u, self.macros)       # (6, N) element energies of the unit strains
                local = -e[3:].sum(0)                   # shear objective density (reproduction.py:137-139)
                w.scal[0] = (local * ls.outer.a.reshape(-1)).mean()
                ls.outer.step_async(local.reshape(ls.outer.x.shape))
                w.scal[1:3].copy_(ls.outer.record())
                w.sh.copy_(w.scal, non_blocking=True)   # x <- new waits for the certificate
            job.end = torch.cuda.Event(enable_timing=True)
            job.end.record(w.stream)

    def _finish(self, w: _Worker, now: float) -> StepResult:
        job = w.job
        info = (_lib.LoadInfo * 6)()
        st = _lib.lib().pgj_solve_wait(w.op._ctx, info, w.stream.cuda_stream)
        if st not in (_lib.PGJ_OK, _lib.PGJ_ERR_CERTIFICATION):
            _lib.check(st, "pgj_solve_wait")
        its = max(i.iterations for i in info)
        lineage = isinstance(job.req, Lineage)
        res = StepResult(tag=job.req.tag, kind="design_step" if lineage else "homogenize",
                         step=job.step, n=w.n, C=w.Ch.numpy().copy(),
                         objective=float(w.sh[0]) if lineage else float("nan"), status=st, iterations=its,
                         queued_ms=(job.admitted - job.ready) * 1e3, latency_ms=(now - job.ready) * 1e3,
                         device_ms=job.start.elapsed_time(job.end),
                         oc_steps=int(w.sh[1]) if lineage else 0, change=float(w.sh[2]) if lineage else 0.0,
                         precision="fp64-fallback" if job.fallback else w.precision)
        w.job = None
        w.last_used = now
        return res

    # ----------------------------------------------------------------------------- loop
    def run(self, arrivals: list[Arrival], realtime: bool = True, idle_sleep: float = 2e-4) -> list[StepResult]:
        """Serve `arrivals` (sorted or not). With realtime=False every request is ready at t=0."""
        pending = deque(sorted(arrivals, key=lambda a: a.t))
        ready: deque[_Job] = deque()
        inflight: list[_Worker] = []
        results: list[StepResult] = []
        t0 = time.perf_counter()
        while pending or ready or inflight:
            now = time.perf_counter()
            while pending and (not realtime or pending[0].t <= now - t0):
                arr = pending.popleft()
                req = arr.req
                if isinstance(req, Lineage) and not supported_n(req.n):
                    raise ValueError(f"unsupported grid size {req.n}")
                ready.append(_Job(req=req, ready=t0 + arr.t if realtime else now,
                                  precision=self._precision_for(req)))
            progressed = False
            # admission in arrival order; a request that cannot start does not block other sizes
            still: deque[_Job] = deque()
            while ready:
                job = ready.popleft()
                w = self._worker_for(self._n_of(job.req), job.precision, self._need(job))
                if w is None:
                    still.append(job)
                    continue
                self._launch(w, job)
                inflight.append(w)
                self.peak_used = max(self.peak_used, self.used)
                progressed = True
            ready = still
            if ready and not inflight and not any(w.job for w in self.workers):
                job = ready[0]
                need = worker_bytes(self._n_of(job.req), job.precision) + self._need(job)
                if need > self.budget:
                    raise RuntimeError(f"request needs {need} bytes, more than the HBM budget {self.budget}")
            self.max_inflight = max(self.max_inflight, len(inflight))
            # completions
            for w in list(inflight):
                if w.job.end.query():
                    now = time.perf_counter()
                    job = w.job
                    res = self._finish(w, now)
                    inflight.remove(w)
                    progressed = True
                    if res.status != 0 and job.precision == "mixed" and self.fallback:
                        # redo in FP64 from the mixed iterate; the design does not advance
                        self.fallbacks += 1
                        redo = _Job(req=job.req, ready=job.ready, lineage=job.lineage, step=job.step,
                                    precision="fp64", fallback=True)
                        if job.lineage is None:
                            redo.u_start = self._snapshot_iterate(w)
                        ready.appendleft(redo)
                        continue
                    results.append(res)
                    if job.lineage is not None:
                        if res.status == 0:
                            job.lineage.pending_advance = True
                        job.lineage.step += 1
                        if job.lineage.step < job.req.steps:
                            ready.append(_Job(req=job.req, ready=now, lineage=job.lineage, step=job.lineage.step,
                                              precision=job.precision))
                        else:
                            self.used -= job.lineage.bytes
            if not progressed:
                if not inflight and not ready and pending and realtime:
                    time.sleep(min(idle_sleep * 10, max(0.0, pending[0].t - (time.perf_counter() - t0))))
                else:
                    time.sleep(idle_sleep)
        self._drain()
        return results


def poisson_lineages(count: int, rate: float, seed: int = 0, n_range=(16, 96), emins=(1e-4, 1e-6, 1e-9),
                     steps: int = 30, **kw) -> list[Arrival]:
    """Poisson arrivals (rate per second) of lineages with n log-uniform over n_range (snapped to a
    supported grid edge) and Emin drawn from emins."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        n = snap_n(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]))))
        emin = float(emins[rng.integers(len(emins))])
        out.append(Arrival(t, Lineage(n=n, seed=1000 + k, emin=emin, steps=steps, tag=k, **kw)))
    return out


def summarize(results: list[StepResult], wall_s: float) -> dict:
    lat = np.array([r.latency_ms for r in results]) if results else np.zeros(1)
    return dict(steps=len(results), wall_s=wall_s, homogenizations_per_s=len(results) / wall_s if wall_s > 0 else 0.0,
                p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                certified=int(sum(1 for r in results if r.status == 0)))
