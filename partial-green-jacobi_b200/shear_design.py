#!/usr/bin/env python
"""Study I periodic shear design (the outer topology-optimization loop over certified solves).

    python partial-green-jacobi_b200/shear_design.py --n 16 --steps 10 --methods 0.5 --output outputs/shear

Same command line, stop rule and output files as the reference's ``examples/shear_design.py:14-74``:
per (method, load mode) a ``Resident`` (three unit shear loads, FP64 PCG certified to 1e-8) starts
from the seeded initial design; each step evaluates the Gaussian-filtered projection at the
staged sharpness beta (1, 2, 4, 8 for 25 steps each), sets the material, selects alpha, solves,
forms the moduli and the energy sensitivity, and runs the OC update. The loop stops after 5
consecutive steps with beta = 8, k >= 95, design change < 0.005 and relative objective change
< 1e-4, or at the step limit. ``<method>_<mode>.json`` holds the per-step rows and
``<method>_<mode>.npz`` the final design ``x`` and ``physical`` density.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

BETA_STAGES = (1.0, 2.0, 4.0, 8.0)
STAGE_STEPS = 25
METHODS = ["green", "gj", "asg", "compact8", "0.5", "0.69"]
TIMING_NOTE = "Demonstration timings include first-use compilation; use registered experiment drivers for benchmarks."


def beta_at(k: int) -> float:
    return BETA_STAGES[min(k // STAGE_STEPS, len(BETA_STAGES) - 1)]


def run(resident, x0, method: str, steps: int, sync=lambda: None) -> tuple[list, bool]:
    """The design loop of one method on ``resident`` from design ``x0``; returns (rows, converged)."""
    resident.outer.set_initial(x0)
    resident.solutions.zero_()
    rows = []
    stable = 0
    for k in range(steps):
        beta = beta_at(k)
        sync()
        start = time.perf_counter()
        resident.outer.evaluate(beta)
        resident.material(resident.outer.a)
        resident.select(method)
        infos, checks = resident.solve()
        moduli, energy = resident.energy()
        resident.outer.step(energy)
        objective = float(moduli.mean())
        change = float(resident.outer.change)
        relative = abs(objective - rows[-1]["objective"]) / abs(objective) if rows else 1.0
        stable = stable + 1 if beta == 8 and k >= 95 and change < 0.005 and relative < 1e-4 else 0
        volume = float(resident.outer.ph.mean())
        sync()
        rows.append(dict(step=k, beta=beta, alpha=float(resident.alpha), objective=objective, volume=volume,
                         change=change, step_s=time.perf_counter() - start, loads=infos, host_checks=checks))
        if stable >= 5 or k == steps - 1:
            break
        resident.outer.advance()
    return rows, stable >= 5


def check_args(n: int, steps: int, methods) -> None:
    if n < 4 or n % 2 or not 1 <= steps <= 180:
        raise ValueError("Use an even n >= 4 and 1 <= steps <= 180.")
    for m in methods:
        if m not in METHODS:
            raise ValueError(f"unknown method {m!r}; choose from {METHODS}")
        if m == "asg" and (n < 32 or n % 16):
            raise ValueError("The ASG selector's features need n >= 32 and n a multiple of 16.")


def main(argv=None):
    p = argparse.ArgumentParser(description="Run the Study I periodic shear design.")
    p.add_argument("--n", type=int, default=16)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--seed", type=int, default=20261104)
    p.add_argument("--methods", nargs="+", default=["0.5"], choices=METHODS)
    p.add_argument("--load-modes", nargs="+", default=["serial"], choices=["serial", "parallel"])
    p.add_argument("--output", type=Path, default=Path("outputs/shear"))
    args = p.parse_args(argv)
    try:
        check_args(args.n, args.steps, args.methods)
    except ValueError as e:
        p.error(str(e))
    import torch

    if not torch.cuda.is_available():
        p.error("A CUDA GPU is required.")
    args.output.mkdir(parents=True, exist_ok=True)
    if any(args.output.iterdir()):
        p.error("Output directory must be empty to preserve prior results.")
    import __graft_entry__ as ge

    pkg = ge.load_package()
    x0 = pkg.study1_initial(args.n, args.seed)
    results = []
    for mode in args.load_modes:
        resident = pkg.Resident(None, args.n, load_mode=mode)
        resident.capture()
        for method in args.methods:
            rows, converged = run(resident, x0, method, args.steps, torch.cuda.synchronize)
            prefix = args.output / f"{method}_{mode}"
            np.savez_compressed(prefix.with_name(prefix.name + ".npz"), x=resident.outer.x.cpu().numpy(),
                                physical=resident.outer.ph.cpu().numpy())
            result = dict(method=method, load_mode=mode, n=args.n, seed=args.seed, optimization_converged=converged,
                          rows=rows, timing_note=TIMING_NOTE)
            prefix.with_name(prefix.name + ".json").write_text(json.dumps(result, indent=2) + "\n")
            results.append(result)
            print(f"{method:8} {mode:8} J={rows[-1]['objective']:.10g} volume={rows[-1]['volume']:.8g} "
                  f"solves={3 * len(rows)}", flush=True)
        del resident
    (args.output / "environment.json").write_text(json.dumps(dict(
        torch=torch.__version__, cuda=torch.version.cuda, gpu=torch.cuda.get_device_name(),
        python=sys.version, command=sys.argv), indent=2) + "\n")
    return results


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    main()
