#!/usr/bin/env python
"""Study II state files (``.npz``) and the preconditioner replay of one state with a warm start.

    python partial-green-jacobi_b200/replay_state.py STATE.npz --eta 1e-6 [--methods gj eta compact8]

Same command line, checks and output record as the reference's ``examples/replay_state.py:14-64``:
the state's ``a`` (stiffness multiplier) and ``rho`` (physical density) are loaded into a
``SelectorResident`` (rmin 3.2, volume 0.2, Emin = eta); for every method the selector and scale are
built, the archived ``u0`` is copied into the solutions, the certified solve runs once to warm up
and once timed, and the record keeps alpha, the per-load infos, the host checks and C_H.

State layout (``docs/DATA.md`` array conventions): scalar fields ``(n, n, n)`` in (z, y, x) order;
``u0`` load-major ``(L, 3 n^3)``, three components per node, L = 6 Voigt loads (xx, yy, zz, yz, xz,
xy) for Study II or 3 shears for Study I. Files are read with ``allow_pickle=False``.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

METHODS = ["green", "gj", "asg", "eta", "contrast", "compact8", "compact8q", "gray"]
ETA_TABLE = (1e-4, 1e-6, 1e-9)
TIMING = ("Selection, preconditioner construction, solve and true residual certification; "
          "one timed repetition.")


def load_state(path) -> dict:
    """Read and check a state file: ``a`` (required), ``rho`` and ``u0`` (optional) as float64."""
    with np.load(path, allow_pickle=False) as z:
        state = {k: np.asarray(z[k]) for k in z.files}
    check_state(state)
    return state


def save_state(path, a, rho=None, u0=None, **extra) -> None:
    """Write a state file in the layout ``load_state`` reads (plain arrays, no pickles)."""
    state = {"a": np.ascontiguousarray(a, dtype=np.float64)}
    if rho is not None:
        state["rho"] = np.ascontiguousarray(rho, dtype=np.float64)
    if u0 is not None:
        state["u0"] = np.ascontiguousarray(u0, dtype=np.float64)
    for k, v in extra.items():
        state[k] = np.asarray(v)
    check_state(state)
    np.savez(path, **state)


def check_state(state: dict) -> None:
    if "a" not in state:
        raise ValueError("state has no 'a' field")
    a = state["a"]
    if a.ndim != 3 or len(set(a.shape)) != 1:
        raise ValueError(f"'a' must be an (n, n, n) field, got shape {a.shape}")
    n = a.shape[0]
    if not np.all(np.isfinite(a)) or a.min() <= 0:
        raise ValueError("'a' must be finite and positive")
    for key in ("rho", "physical", "x"):
        if key in state and state[key].shape != a.shape:
            raise ValueError(f"'{key}' must have the shape of 'a' {a.shape}, got {state[key].shape}")
    for key in ("u0", "previous", "solution"):
        if key in state:
            u = state[key]
            if u.ndim != 2 or u.shape[1] != 3 * n ** 3 or u.shape[0] not in (3, 6):
                raise ValueError(f"'{key}' must be load-major (3 or 6, 3 n^3) = (L, {3 * n ** 3}), got {u.shape}")


def check_methods(methods, eta) -> None:
    """The reference CLI's checks: known methods or an exponent in [0, 1], no ASG, a calibrated eta."""
    for method in methods:
        if method not in METHODS:
            try:
                if not 0 <= float(method) <= 1:
                    raise ValueError()
            except ValueError:
                raise ValueError("Unknown method or exponent outside [0,1]: " + str(method)) from None
        if method == "asg":
            raise ValueError("Frozen ASG belongs to Study I; use examples/shear_design.py.")
    if eta not in ETA_TABLE:
        raise ValueError("The calibrated eta table supports 1e-4, 1e-6 and 1e-9.")


def _device_resident(n, objective, eta, load_mode):
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    r = pkg.SelectorResident(None, n, objective, 0.2, rmin=3.2, emin=eta, load_mode=load_mode)
    r.capture()
    return r, (lambda x: torch.as_tensor(x, device="cuda")), torch.cuda.synchronize


def replay(state: dict, eta: float, objective: str = "shear", load_mode: str = "parallel",
           methods=("gj", "eta", "compact8"), resident=None) -> list:
    """Replay ``state`` for each method; returns the per-method records.

    ``resident`` = (resident, to_device, synchronize) overrides the device resident (tests).
    """
    check_methods(methods, eta)
    check_state(state)
    if "rho" not in state or "u0" not in state:
        raise ValueError("replay needs the state's 'rho' and 'u0' fields")
    n = state["a"].shape[0]
    r, dev, sync = resident or _device_resident(n, objective, eta, load_mode)
    r.material(dev(state["a"]))
    r.outer.ph.copy_(dev(state["rho"]))
    u0 = dev(state["u0"])
    records = []
    for method in methods:
        # warm each method, then reset the identical archived initial guess
        r.select(method)
        r.solutions.copy_(u0)
        r.solve()
        r.solutions.copy_(u0)
        sync()
        start = time.perf_counter()
        r.select(method)
        loads, checks = r.solve()
        sync()
        elapsed = time.perf_counter() - start
        records.append(dict(method=method, alpha=float(r.alpha), analysis_s=elapsed, loads=loads,
                            host_checks=checks, C=r.effective_tensor().cpu().tolist()))
        print(method, elapsed, "s", flush=True)
    return records


def main(argv=None):
    p = argparse.ArgumentParser(description="Compare preconditioners on one Study II state and warm start.")
    p.add_argument("state", type=Path)
    p.add_argument("--eta", type=float, required=True)
    p.add_argument("--objective", choices=["shear", "bulk", "auxetic"], default="shear")
    p.add_argument("--load-mode", choices=["serial", "parallel"], default="parallel")
    p.add_argument("--methods", nargs="+", default=["gj", "eta", "compact8"])
    p.add_argument("--output", type=Path, default=Path("outputs/replay.json"))
    a = p.parse_args(argv)
    try:
        check_methods(a.methods, a.eta)
    except ValueError as e:
        p.error(str(e))
    if a.output.exists():
        p.error("Output exists; choose a new path.")
    records = replay(load_state(a.state), a.eta, a.objective, a.load_mode, a.methods)
    a.output.parent.mkdir(parents=True, exist_ok=True)
    a.output.write_text(json.dumps(dict(state=a.state.name, eta=a.eta, load_mode=a.load_mode, timing=TIMING,
                                        records=records), indent=2) + "\n")


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    main()
