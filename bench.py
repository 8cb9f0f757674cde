#!/usr/bin/env python
"""Certified 6-load homogenizations/s (p50/p99 latency), mixed vs FP64, on B200.

Workload (one homogenization): a seeded synthetic design at n=64 (N(0,1) noise, periodic Gaussian
sigma=n/16, quantile threshold to vf=0.35, logistic width 0.1; SIMP p=3, E0=1, Emin=1e-6; paper
medium E=1, nu=0.3), the six unit Voigt loads as parallel PCG recurrences from a zero start, partial
Green-Jacobi alpha=0.5, every load certified to relative true residual <= 1e-8 by the FP64 true
residual, then C_H (6x6).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pgj|reference]

* value        headline: batched mixed precision (FP32 inner PCG, FP64 reliable updates and FP64
               certificate), `slots` batched contexts of `designs` designs each (one kernel launch
               carries all designs of a context); one step = one homogenization of every in-flight
               design (slots * designs); designs resident in HBM; CUDA events on the streams.
* fp64         the plain FP64 drop-in, one design at a time (the reference's recurrence), and the
               batched FP64 path, beside the headline; mixed single-design too.
* e2e          the headline path through the public API (pgj_b200.Batch) with every design copied
               from pinned host memory and C_H copied back inside the timed region.
* roofline     dominant kernel of the headline path's PCG iteration, timed live with CUDA events on a
               batched context (pgj_profile_iteration), against the measured HBM copy bandwidth.
* uneven       64 designs (seeds 0..63) with n from {24, 32, 48, 64}, vf in [0.2, 0.5], alpha in
               [0, 1], batched by grid size, FP64 and mixed, each certified to 1e-8.
* cpu_baseline the CPU restatement of the reference arithmetic (oracle/pgj_oracle.py): one complete
               n=16 homogenization with serial loads, plus a bounded n=64 sample extrapolated to the
               oracle's own certified iteration count (tests/golden/config2.json).
* serving      continuous batching (pgj_b200.serve): Poisson arrivals of design lineages with n
               log-uniform over [16, 96] and Emin in {1e-4, 1e-6, 1e-9}; each design step is a
               warm-started certified homogenization, the shear sensitivity and the OC update
               (move 0.2, filter radius 1.5) on the device; throughput and p50/p99 step latency on
               the host clock per offered load, mixed and plain FP64 servers on the same arrivals.
Multi-GPU: replicas only (independent designs per rank, no collective on the data path); the
timing is max-over-ranks; value = all homogenizations / that time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "certified 6-load homogenizations/s & p50/p99 latency, mixed vs FP64 at 1e-8"
UNIT = "homogenizations/s"
N_GRID, EMIN, ALPHA, RTOL, NSEEDS = 64, 1e-6, 0.5, 1e-8, 8
FALLBACK_HBM = 6650.0
L2_BYTES = 126e6


def oracle_iterations(n=N_GRID, emin=EMIN, alpha=ALPHA, seed=0):
    """Certified FP64 PCG iterations of the CPU oracle on this workload (max over the six loads),
    from the committed fixture tests/golden/config2.json (tests/golden/make_config2.py)."""
    p = ROOT / "tests" / "golden" / "config2.json"
    if p.exists():
        rec = json.loads(p.read_text())["cases"].get(f"n{n}/a{alpha:g}/e{emin:g}/s{seed}")
        if rec:
            return int(max(rec["iterations"])), f"oracle fixture n{n}/a{alpha:g}/e{emin:g}/s{seed}"
    return None, "no oracle fixture"


def workload_config(arith, extra=None):
    cfg = {"workload": f"periodic HEX8 homogenization n={N_GRID}, 6 Voigt loads parallel, {arith}, "
                       f"alpha={ALPHA}, Emin={EMIN:g}, zero start, rtol={RTOL:g} (FP64 true residual), C_H",
           "n": N_GRID, "loads": 6, "emin": EMIN, "alpha": ALPHA, "rtol": RTOL, "vf": 0.35,
           "designs": f"seeds rank*1000+0..{NSEEDS - 1}, cycled", "medium": "E=1, nu=0.3",
           "l2": "working set per homogenization ~310 MB > 126 MB L2 (no flush needed)",
           "parallelism": "replicas"}
    if extra:
        cfg.update(extra)
    return cfg


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(kernel, prec):
    """DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` at n=64."""
    p = ROOT / "profiles" / "traffic_n64.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(prec, {}).get(kernel)
    return None


# ------------------------------------------------------------------------------------------ CPU
def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import pgj_oracle as O

    return O


def cpu_complete_config1(seed=0):
    """One complete CPU homogenization of the n=16 configuration (serial loads: one recurrence per
    Voigt load, one after the other; alpha 0.5, Emin 1e-6, zero start, rtol 1e-8, C_H), timed
    end to end without extrapolation."""
    O = _oracle()
    from __graft_entry__ import load_package

    n = 16
    a = load_package().baseline_design(n, seed, EMIN)
    lam, mu = O.PAPER
    t0 = time.perf_counter()
    prob = O.Problem(a, lam, mu, ALPHA)
    f = O.rhs(prob.a, np.eye(6), lam, mu)
    u = np.zeros_like(f)
    its = []
    for l in range(6):
        ul, infos, raised = O.solve_batch(prob, f[l:l + 1])
        u[l] = ul[0]
        its.append(infos[0].iterations)
        if raised:
            raise RuntimeError(("CPU config-1 certification failed", infos))
    O.effective_tensor(prob.a, u, lam, mu)
    sec = time.perf_counter() - t0
    return dict(n=n, seconds=sec, value=1.0 / sec, iterations=its, loads="serial")


def cpu_sample(n=N_GRID, seed=0, iters=4, its_full=None):
    """Oracle timing sample at n=64: setup + `iters` PCG iterations + one energy evaluation,
    extrapolated to `its_full` certified iterations and the 21 energy evaluations of C_H."""
    O = _oracle()
    from __graft_entry__ import load_package

    a = load_package().baseline_design(n, seed, EMIN)
    lam, mu = O.PAPER
    t0 = time.perf_counter()
    prob = O.Problem(a, lam, mu, ALPHA)
    f = O.rhs(prob.a, np.eye(6), lam, mu)
    t1 = time.perf_counter()
    u, infos, _ = O.solve_batch(prob, f, max_iterations=0)  # certification + init only
    t2 = time.perf_counter()
    O.solve_batch(prob, f, max_iterations=iters)
    t3 = time.perf_counter()
    aff = O.affine(n, np.eye(6))
    O.energies(u[:1], aff[:1], n, lam, mu)
    t4 = time.perf_counter()
    per_iter = max((t3 - t2) - (t2 - t1), 1e-9) / iters
    setup = (t1 - t0) + (t2 - t1)  # problem setup, rhs, certification + initialisation + final certification
    total = setup + its_full * per_iter + 21 * (t4 - t3)  # C_H by polarisation: 21 single-load energy evaluations
    return dict(value=1.0 / total, seconds_per_homogenization=total, per_iteration_s=per_iter, setup_s=setup,
                energy_s=(t4 - t3), iterations=its_full)


# ------------------------------------------------------------------------------------------ GPU
def design_seeds(rank, count=NSEEDS):
    """Replicas only: every rank homogenizes its own designs (disjoint seeds), no data exchange."""
    return [rank * 1000 + k for k in range(count)]


def designs_for(rank, pkg):
    return [pkg.baseline_design(N_GRID, s, EMIN) for s in design_seeds(rank)]


def run_single(args, pkg, dev, prec, stream, local_rank, world):
    """The one-design path (Operator.solve + C_H per homogenization), K timed steps."""
    import torch

    lam, mu = pkg.PAPER_MEDIUM
    eye6 = np.eye(6)
    u = torch.zeros((6, 3 * N_GRID ** 3), dtype=torch.float64, device="cuda")
    op = pkg.Operator(N_GRID, 6, lam, mu, precision=prec)
    iters, launches, sweeps, tensors = [], [], [], []

    def step(k, record=True):
        op.set_material(dev[k % len(dev)])
        op.set_alpha(ALPHA)
        u.zero_()
        infos, st = op.solve(eye6, RTOL, u)
        if st != 0:
            raise RuntimeError(("certification failed", prec, infos))
        C = op.effective_tensor(u)
        if record:
            iters.append([i["iterations"] for i in infos])
            launches.append(op.last_launches() + 3)  # + scale build (2) + C_H (1)
            sweeps.append(op.last_refinements())
            tensors.append(C)

    for k in range(args.warmup):
        step(k, record=False)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local_rank) as clocks:
        ev[0].record(stream)
        for k in range(args.steps):
            step(k)
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    lat = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    out = dict(total_ms=ev[0].elapsed_time(ev[-1]), lat=lat, iters=iters, launches=launches, sweeps=sweeps,
               clocks=clocks.summary(), tiles=op.tile_shapes(), homs=args.steps,
               C=[C.cpu().numpy() for C in tensors])
    out["prof"] = op.profile_iteration(eye6, reps=20)
    torch.cuda.synchronize()
    return out


def timed_batch(args, pkg, batch, inputs, count, local_rank, world):
    """Run `count` requests through `batch` after a warm-up; device time from the first launch to
    the last stream's completion."""
    import torch

    def reqs(k, tag0=0):
        return [pkg.Request(inputs[(tag0 + i) % len(inputs)], ALPHA, tag=tag0 + i) for i in range(k)]

    batch.run(reqs(args.warmup * batch.slots * batch.designs))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    main = torch.cuda.current_stream()
    t0 = torch.cuda.Event(enable_timing=True)
    t0.record(main)
    for st in batch.streams():
        st.wait_event(t0)
    with ClockSampler(local_rank) as clocks:
        res = batch.run(reqs(count))
        ends = []
        for st in batch.streams():
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(st)
            ends.append(ev)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    bad = [r for r in res if r.status != 0]
    if bad:
        raise RuntimeError(("batched certification failed", bad[0].infos))
    return max(t0.elapsed_time(ev) for ev in ends), res, clocks.summary()


def run_uneven(args, pkg, count):
    """The uneven batch: `count` designs (n from {24, 32, 48, 64}), batched by grid size."""
    import torch

    designs = pkg.designs.uneven_designs(count, EMIN)
    out = {}
    for prec in ("mixed", "fp64"):
        batch = pkg.Batch(slots=args.slots, designs=args.designs, precision=prec)
        for n in sorted({d[1] for d in designs}):
            batch.warm(n)
        dev = {seed: torch.tensor(a, device="cuda") for seed, n, vf, alpha, a in designs}
        reqs = [pkg.Request(dev[seed], alpha, tag=seed) for seed, n, vf, alpha, a in designs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = batch.run(reqs)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ok = [r for r in res if r.status == 0]
        out[prec] = {"designs": len(res), "certified": len(ok), "seconds": wall,
                     "homogenizations_per_s": len(res) / wall,
                     "certified_per_s": len(ok) / wall,
                     "uncertified": sorted(r.tag for r in res if r.status != 0),
                     "iterations_per_load_mean": float(np.mean([[i["iterations"] for i in r.infos] for r in res])),
                     "C": {r.tag: r.C for r in res}}
        del batch
        torch.cuda.empty_cache()
    errs = [float(np.abs(out["mixed"]["C"][t] - out["fp64"]["C"][t]).max() / np.abs(out["fp64"]["C"][t]).max())
            for t in out["fp64"]["C"] if t in out["mixed"]["C"]]
    for prec in out:
        out[prec].pop("C")
    out["mixed"]["ch_rel_err_vs_fp64_max"] = max(errs) if errs else None
    out["config"] = {"count": count, "grids": "uniform over {24, 32, 48, 64}", "vf": "uniform [0.2, 0.5]",
                     "alpha": "uniform [0, 1]", "emin": EMIN, "sigma": "n/16", "seeds": f"0..{count - 1}",
                     "timing": "host wall clock around Batch.run (all designs resident in HBM), one pass",
                     "batching": f"{args.slots} batched contexts x {args.designs} designs per grid size"}
    return out


def run_gpu(args, rank, world, local_rank):
    import torch

    from __graft_entry__ import load_package

    pkg = load_package()
    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream()
    host = designs_for(rank, pkg)
    out = {}
    with torch.cuda.stream(stream):
        dev = [torch.tensor(a, device="cuda") for a in host]
        for prec in ("mixed", "fp64"):
            out[prec] = run_single(args, pkg, dev, prec, stream, local_rank, world)
    errs = [float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(out["mixed"]["C"], out["fp64"]["C"])]
    out["mixed"]["ch_rel_err_vs_fp64"] = max(errs)
    ref_C = out["fp64"]["C"]

    # batched paths: slots x designs in flight; one step = one homogenization of each
    per_step = args.slots * args.designs
    for prec in ("mixed", "fp64"):
        batch = pkg.Batch(slots=args.slots, designs=args.designs, precision=prec)
        batch.warm(N_GRID)
        total, res, clocks = timed_batch(args, pkg, batch, dev, args.steps * per_step, local_rank, world)
        leg = dict(total_ms=total, lat=[r.latency_ms for r in res], homs=len(res),
                   iters=[[i["iterations"] for i in r.infos] for r in res], launches=[r.launches for r in res],
                   clocks=clocks, sweeps=[r.refinements for r in res])
        errs = [float(np.abs(r.C - ref_C[r.tag % len(dev)]).max() / np.abs(ref_C[r.tag % len(dev)]).max())
                for r in res if r.tag % len(dev) < len(ref_C)]
        leg["ch_rel_err_vs_fp64"] = max(errs) if errs else None
        if prec == "mixed":
            pinned = [torch.from_numpy(a).pin_memory() for a in host]
            leg["e2e_ms"], _, _ = timed_batch(args, pkg, batch, pinned, args.steps * per_step, local_rank, world)
            # roofline of the headline path: one batched context with all its designs' loads
            bop = batch.pool[N_GRID][0].op
            for d in range(args.designs):
                bop.set_material(d, dev[d % len(dev)], torch.cuda.current_stream())
                bop.set_alpha(d, ALPHA, torch.cuda.current_stream())
            leg["prof"] = bop.profile_iteration(np.eye(6), reps=20)
            leg["tiles"] = bop.tile_shapes()
        out[f"batched_{prec}"] = leg
        del batch
        torch.cuda.empty_cache()

    if world > 1:
        keys = ["mixed", "fp64", "batched_mixed", "batched_fp64"]
        t = torch.tensor([out[k]["total_ms"] for k in keys] + [out["batched_mixed"]["e2e_ms"]], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        for i, k in enumerate(keys):
            out[k]["total_ms"] = float(t[i])
        out["batched_mixed"]["e2e_ms"] = float(t[-1])
    out["h2d"] = host[0].nbytes
    out["d2h"] = 36 * 8
    if rank == 0 and args.uneven > 0:
        out["uneven"] = run_uneven(args, pkg, args.uneven)
    if args.serve_lineages > 0 and rank == 0:
        out["serving"] = run_serving(args, pkg)
    return out


def run_serving(args, pkg):
    """Continuous batching of design lineages, mixed and plain FP64 servers on the same arrivals,
    at each offered load (lineage arrival rate) of the sweep."""
    sv = pkg.serve
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    out = {"config": {"lineages": args.serve_lineages, "steps_per_lineage": args.serve_steps,
                      "arrival_rates_per_s": rates, "hbm_budget_gb": 120, "move": 0.2, "rmin": 1.5,
                      "volume": 0.3, "alpha": ALPHA, "objective": "shear",
                      "n": "log-uniform over [16, 96], snapped to supported even 5-smooth sizes",
                      "emin": "uniform over {1e-4, 1e-6, 1e-9}",
                      "latency": "host clock, step ready -> C_H and OC record on the host (queueing included)"},
           "sweep": []}
    for rate in rates:
        arrivals = sv.poisson_lineages(args.serve_lineages, rate, seed=11, steps=args.serve_steps)
        point = {"arrival_rate_per_s": rate, "n": [a.req.n for a in arrivals], "emin": [a.req.emin for a in arrivals]}
        for prec in ("mixed", "fp64"):
            # contexts of every grid size once first, so the tile autotuners stay outside the timed run
            for n in sorted({a.req.n for a in arrivals}):
                for p in {prec, "fp64"}:
                    pkg.Operator(n, 6, *pkg.PAPER_MEDIUM, precision=p)
            server = sv.Server(precision=prec, hbm_budget=120e9)
            server.warm([a.req for a in arrivals])  # workers and their solve graphs outside the timed run
            t0 = time.perf_counter()
            res = server.run(arrivals, realtime=True)
            wall = time.perf_counter() - t0
            st = sv.summarize(res, wall)
            st.update(max_in_flight=server.max_inflight, peak_hbm_gb=server.peak_used / 1e9,
                      iterations_mean=float(np.mean([r.iterations for r in res])), fallbacks=server.fallbacks,
                      steps_by_precision={k: sum(1 for r in res if r.precision == k)
                                          for k in sorted({r.precision for r in res})})
            point[prec] = st
        point["over_plain_fp64"] = point["mixed"]["homogenizations_per_s"] / point["fp64"]["homogenizations_per_s"]
        out["sweep"].append(point)
    return out


def roofline(prof, hbm, kind, prec):
    dom = max(prof, key=lambda k: prof[k]["ms"])
    achieved = prof[dom]["bytes"] / (prof[dom]["ms"] * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": kind, "algorithmic_bytes": prof[dom]["bytes"],
            "traffic": traffic_from_profiles(dom, prec),
            "iteration_ms": sum(v["ms"] for v in prof.values()),
            "kernels": {k: {"ms": v["ms"], "GBps": v["bytes"] / (v["ms"] * 1e-3) / 1e9} for k, v in prof.items()}}


def reference_arm(args, rank):
    """The reference's CPU implementation of the path (the oracle port: the reference has no CPU solver)
    on this host's cores: per step, one complete n=16 homogenization (serial loads) and a bounded n=64
    sample extrapolated to the oracle's certified iteration count of the headline workload."""
    if rank != 0:
        return
    its, its_src = oracle_iterations()
    if its is None:
        raise RuntimeError("tests/golden/config2.json lacks the n=64 oracle record")
    samples, complete = [], []
    t_start = time.perf_counter()
    for k in range(args.warmup + args.steps):
        s = cpu_sample(seed=0, iters=2, its_full=its)
        c = cpu_complete_config1(seed=k % 3)
        if k >= args.warmup:
            samples.append(s)
            complete.append(c)
    value = float(np.mean([s["value"] for s in samples]))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config("FP64 PCG (CPU oracle port)",
                                      {"extrapolation": f"per-step sample: setup + 2 PCG iterations + 1 energy "
                                                        f"evaluation, scaled to {its} iterations ({its_src}: the "
                                                        "oracle's certified FP64 count) and 21 energy evaluations"}),
            "impl": "reference",
            "config1_complete": {"what": "one complete CPU homogenization per step, n=16, serial loads, alpha 0.5, "
                                         "Emin 1e-6, rtol 1e-8, C_H (no extrapolation)",
                                 "homogenizations_per_s": float(np.mean([c["value"] for c in complete])),
                                 "seconds": [c["seconds"] for c in complete],
                                 "iterations": [c["iterations"] for c in complete]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": "CPU restatement of the reference arithmetic (NumPy/SciPy, all host threads "
                                       "for the FFTs); per step a bounded n=64 sample extrapolated to one "
                                       "homogenization, beside one complete n=16 homogenization"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t_start}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["pgj", "reference"], default="pgj")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--slots", type=int, default=2, help="batched contexts in flight (one stream each)")
    ap.add_argument("--designs", type=int, default=4, help="designs per batched context (one launch carries all)")
    ap.add_argument("--uneven", type=int, default=64, help="designs of the uneven batch leg (0: skip)")
    ap.add_argument("--serve-lineages", type=int, default=6, help="design lineages per serving run (0: skip)")
    ap.add_argument("--serve-steps", type=int, default=30, help="design steps per lineage in the serving leg")
    ap.add_argument("--serve-rates", default="0.5,2,8", help="lineage arrival rates per second (Poisson), swept")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch

    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_gpu(args, rank, world, local_rank)
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    hbm, kind = peaks()

    def summary(d):
        lat = sorted(d["lat"])
        its = np.array(d["iters"])
        homs = d["homs"] * world
        return {"value": homs / (d["total_ms"] / 1000.0), "ms_per_step": d["total_ms"] / args.steps,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "iterations_per_load_mean": float(its.mean()), "iterations_max_mean": float(its.max(1).mean())}

    mx, f64 = summary(res["mixed"]), summary(res["fp64"])
    bt, bf = summary(res["batched_mixed"]), summary(res["batched_fp64"])
    bm = res["batched_mixed"]
    e2e = bm["homs"] * world / (bm["e2e_ms"] / 1000.0)
    its_oracle, its_src = oracle_iterations()
    line = {"metric": METRIC, "value": bt["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": bt["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (FP32 inner PCG, FP64 true residual)",
            "data": "synthetic",
            "config": workload_config("batched mixed precision (FP32 inner PCG, FP64 reliable updates, FP64 "
                                      "certificate)",
                                      {"path": f"{args.slots} batched contexts x {args.designs} designs in flight "
                                               "(each context: one graph launch per certified solve of all its "
                                               "designs); one step = one homogenization of each of the "
                                               f"{args.slots * args.designs} designs",
                                       "slots": args.slots, "designs_per_context": args.designs}),
            "p50_ms": bt["p50_ms"], "p99_ms": bt["p99_ms"],
            "iterations_per_load_mean": bt["iterations_per_load_mean"],
            "refinements_mean": float(np.mean(bm["sweeps"])),
            "ch_rel_err_vs_fp64": bm["ch_rel_err_vs_fp64"],
            "over_plain_fp64": bt["value"] / f64["value"],
            "fp64": dict(f64, roofline=roofline(res["fp64"]["prof"], hbm, kind, "fp64"), clocks=res["fp64"]["clocks"],
                         tiles=res["fp64"]["tiles"], oracle_iterations=its_oracle, oracle_source=its_src),
            "fp64_batched": dict(bf, ch_rel_err_vs_fp64=res["batched_fp64"]["ch_rel_err_vs_fp64"]),
            "mixed_single": dict(mx, ch_rel_err_vs_fp64=res["mixed"]["ch_rel_err_vs_fp64"],
                                 roofline=roofline(res["mixed"]["prof"], hbm, kind, "mixed")),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": res["h2d"] * args.slots * args.designs,
                    "d2h_bytes_per_step": res["d2h"] * args.slots * args.designs},
            "roofline": roofline(bm["prof"], hbm, kind, "mixed_batched"), "tiles": bm["tiles"],
            "gpu_launches": int(sum(bm["launches"])), "clocks": bm["clocks"]}
    if "uneven" in res:
        line["uneven"] = res["uneven"]
    if "serving" in res:
        line["serving"] = res["serving"]
    if world == 1 and not args.no_cpu:
        its = its_oracle or int(round(f64["iterations_max_mean"]))
        cb = cpu_sample(its_full=its)
        c1 = cpu_complete_config1()
        line["cpu_baseline"] = {"value": cb["value"], "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                "sample": f"oracle n=64 6 loads FP64: setup + 4 PCG iterations + 1 energy "
                                          f"evaluation, extrapolated to {cb['iterations']} iterations ({its_src}) "
                                          f"and 21 energies; {cb['per_iteration_s']:.3f} s/iteration",
                                "config1_complete": {"n": 16, "loads": "serial", "seconds": c1["seconds"],
                                                     "homogenizations_per_s": c1["value"],
                                                     "iterations": c1["iterations"]}}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
