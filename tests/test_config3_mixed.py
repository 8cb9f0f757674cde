"""Mixed-precision refinement on the large grids: n = 96 and 128, Emin/E0 in {1e-6, 1e-9}, alpha 0.5,
seeded baseline design (seed 0), six Voigt loads from a zero start.

The form is the refinement one: FP32 PCG (FP32 operator, FP32 Green apply) to an inner relative
tolerance of 1e-5 per sweep, the correction accumulated into the FP64 iterate, and the FP64 true
residual f - K u certifying every load to 1e-8 (`set_mixed_mode("sweeps")`, iteration cap 8000 per
sweep: at Emin 1e-9 the FP32 recurrence needs more iterations than the FP64 drop-in's 4000).

Bars, per case: the FP64 drop-in and the refinement both certify; the refinement takes between 1 and
12 sweeps; C_H of the refinement is within 1e-7 of the FP64 solve, and, where the CPU oracle's fixture
for the case exists (tests/golden/config3.json, written by tests/golden/make_config2.py --set config3),
within 1e-7 of the oracle, with the FP64 solve within 1e-10 of it. Each case's sweeps, iteration
counts and errors are appended to the JSON-lines file named by PGJ_CONFIG3_LOG, when set.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "config3.json"
ORACLE = json.loads(FIXTURE.read_text())["cases"] if FIXTURE.exists() else {}

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes, skipped
    pytest.skip("CUDA device required", allow_module_level=True)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("n,emin", [(96, 1e-6), (96, 1e-9), (128, 1e-6), (128, 1e-9)])
def test_refinement_certifies_and_matches_fp64(pkg, n, emin):
    lam, mu = pkg.PAPER_MEDIUM
    a = torch.tensor(pkg.baseline_design(n, 0, emin), device="cuda")
    res = {}
    for prec in ("fp64", "mixed"):
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        if prec == "mixed":
            op.set_mixed_mode("sweeps")
            op.set_inner_rtol(1e-5)
            op.set_iteration_cap(8000)
        op.set_material(a)
        op.set_alpha(0.5)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0 and all(i["converged"] and i["relative_residual"] <= 1e-8 for i in infos), (prec, infos)
        res[prec] = dict(C=op.effective_tensor(u).cpu().numpy(), sweeps=op.last_refinements(),
                         iterations=[i["iterations"] for i in infos])
        del op, u
        torch.cuda.empty_cache()
    sweeps = res["mixed"]["sweeps"]
    assert 1 <= sweeps <= 12, sweeps
    err = rel(res["mixed"]["C"], res["fp64"]["C"])
    assert err <= 1e-7, err
    key = f"n{n}/a0.5/e{emin:g}/s0"
    rec = dict(key=key, sweeps=sweeps, iterations_mixed=res["mixed"]["iterations"],
               iterations_fp64=res["fp64"]["iterations"], ch_mixed_vs_fp64=err)
    if key in ORACLE and not ORACLE[key]["raised"]:
        C = ORACLE[key]["C"]
        rec["ch_fp64_vs_oracle"] = rel(res["fp64"]["C"], C)
        rec["ch_mixed_vs_oracle"] = rel(res["mixed"]["C"], C)
        assert rec["ch_fp64_vs_oracle"] <= 1e-10, rec
        assert rec["ch_mixed_vs_oracle"] <= 1e-7, rec
    path = os.environ.get("PGJ_CONFIG3_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(rec) + "\n")
