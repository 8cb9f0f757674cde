"""FP64 drop-in parity on the benchmark grid against the CPU oracle's fixtures (tests/golden/config2.json,
written by tests/golden/make_config2.py).

Cases: n = 32 over alpha in {0, 0.5, 1} x Emin/E0 in {1e-4, 1e-6, 1e-9} x seeds 0..4, and n = 64 at
alpha = 0.5 x Emin/E0 in {1e-4, 1e-6, 1e-9}, seed 0; six Voigt loads, zero start, rtol 1e-8.

Bars, per case:
* C_H of the FP64 path within 1e-10 relative of the oracle's (max entry), when the oracle certified;
* iteration counts, per load: equal to the oracle's for pure Green (alpha = 0: no diagonal scaling;
  every load of the 15 cases, capped or not, matches exactly), within max(1, 2%) for alpha = 0.5 and
  within max(1, 4%) for alpha = 1. With the scaling D^-alpha/2 the counts of this ill-conditioned PCG
  depend on rounding-level differences of the arithmetic: the device's counts are systematically
  lower than the oracle's, by up to 1.1% at alpha = 0.5 and 2.9% at alpha = 1 (Emin 1e-9), while the
  oracle's two summation orders agree within a few iterations and its run with the reference's own
  modal element arithmetic moves in the device's direction; the reference itself moves by 1.7%
  between its two schedules (582 vs 592 in exp/asg_mutopopt_20261104/results/replay_n64_k062.json).
  Each case's counts are appended to the JSON-lines file named by PGJ_DELTA_LOG, when set;
* a case the oracle could not certify (pure Green, alpha = 0, at high contrast hits the 4000-iteration
  cap) must be reported uncertified by the device too;
* the mixed path (FP32 inner recurrence, FP64 certificate, iteration cap 8000) certifies the
  alpha = 0.5 cases with C_H within 1e-7 of the oracle.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "config2.json"
CASES = json.loads(FIXTURE.read_text())["cases"] if FIXTURE.exists() else {}

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes, skipped
    pytest.skip("CUDA device required", allow_module_level=True)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def count_ok(dev, ref, alpha):
    if alpha == 0.0:
        return dev == ref
    frac = 0.02 if alpha <= 0.5 else 0.04
    return abs(dev - ref) <= max(1, int(np.ceil(frac * ref)))


def log_deltas(key, precision, its, rec, st):
    path = os.environ.get("PGJ_DELTA_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(dict(key=key, precision=precision, device=its, oracle=rec["iterations"],
                                     oracle_b=rec["iterations_b"], oracle_r=rec.get("iterations_r"), status=st,
                                     oracle_raised=rec["raised"])) + "\n")


def solve(pkg, rec, precision):
    n, alpha, emin, seed = rec["n"], rec["alpha"], rec["emin"], rec["seed"]
    op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM, precision=precision)
    if precision == "mixed":
        # the FP32 recurrence takes more (cheaper) iterations at high contrast: n = 64, Emin 1e-9,
        # alpha 0.5 certifies at about 4300; the FP64 drop-in keeps the reference's 4000
        op.set_iteration_cap(8000)
    op.set_material(torch.tensor(pkg.baseline_design(n, seed, emin), device="cuda"))
    op.set_alpha(alpha)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    C = op.effective_tensor(u).cpu().numpy()
    return infos, st, C


@pytest.mark.skipif(not CASES, reason="oracle fixture tests/golden/config2.json absent")
@pytest.mark.parametrize("key", sorted(CASES))
def test_fp64_dropin_matches_oracle(pkg, key):
    rec = CASES[key]
    infos, st, C = solve(pkg, rec, "fp64")
    its = [i["iterations"] for i in infos]
    log_deltas(key, "fp64", its, rec, st)
    if rec["raised"]:
        assert st == pkg._lib.PGJ_ERR_CERTIFICATION, (key, its)
        assert its == rec["iterations"], (key, its, rec["iterations"])  # the cap, load by load
        return
    assert st == 0, (key, infos)
    assert rel(C, rec["C"]) <= 1e-10, (key, rel(C, rec["C"]))
    for l, (d, a) in enumerate(zip(its, rec["iterations"])):
        assert count_ok(d, a, rec["alpha"]), (key, l, its, rec["iterations"], rec["iterations_b"])


@pytest.mark.skipif(not CASES, reason="oracle fixture tests/golden/config2.json absent")
@pytest.mark.parametrize("key", sorted(k for k in CASES if CASES[k]["alpha"] == 0.5))
def test_mixed_matches_oracle(pkg, key):
    rec = CASES[key]
    if rec["raised"]:
        pytest.skip("the oracle did not certify this case")
    infos, st, C = solve(pkg, rec, "mixed")
    log_deltas(key, "mixed", [i["iterations"] for i in infos], rec, st)
    assert st == 0, (key, infos)
    assert all(i["relative_residual"] <= 1e-8 for i in infos)
    assert rel(C, rec["C"]) <= 1e-7, (key, rel(C, rec["C"]))
