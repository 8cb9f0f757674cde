"""CPU checks of the benchmark-grid oracle fixtures (tests/golden/config2.json, config3.json), which the
GPU parity tests hold the device to: well-formed records, physically sane tensors, the two summation
orders of the oracle within a few iterations of each other, and one case re-solved here by the oracle
with the same counts and C_H (the fixture is what the committed oracle computes)."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def cases(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip(f"{name} absent")
    return json.loads(p.read_text())["cases"]


@pytest.mark.parametrize("name", ["config2.json", "config3.json"])
def test_records_are_well_formed(name):
    for key, r in cases(name).items():
        n, alpha, emin, seed = r["n"], r["alpha"], r["emin"], r["seed"]
        assert key == f"n{n}/a{alpha:g}/e{emin:g}/s{seed}"
        assert len(r["iterations"]) == 6 and len(r["relative_residual"]) == 6
        assert r["raised"] == (not all(r["converged"])), key
        if r["raised"]:
            assert max(r["iterations"]) == 4000, key  # an uncertified oracle run ends at the iteration cap
            continue
        assert max(r["relative_residual"]) <= 1e-8, key
        C = np.asarray(r["C"])
        assert np.abs(C - C.T).max() <= 1e-10 * np.abs(C).max(), key
        assert np.linalg.eigvalsh(0.5 * (C + C.T)).min() > 0, key


def test_summation_orders_agree_within_a_few_iterations():
    worst = 0
    for key, r in cases("config2.json").items():
        if r["iterations_b"] is None:
            continue
        for a, b in zip(r["iterations"], r["iterations_b"]):
            worst = max(worst, abs(a - b))
            assert abs(a - b) <= max(3, 0.01 * a), (key, r["iterations"], r["iterations_b"])
        if not r["raised"]:
            assert np.abs(np.subtract(r["C"], r["C_b"])).max() <= 1e-10 * np.abs(r["C"]).max(), key
    assert worst <= 7


def test_one_case_resolves_to_the_fixture(oracle):
    r = cases("config2.json")["n32/a0.5/e0.0001/s3"]
    a = oracle.simp(oracle.baseline_density(32, 3), 1e-4)
    res = oracle.homogenize(a, *oracle.PAPER, 0.5, rtol=1e-8)
    assert [i.iterations for i in res["infos"]] == r["iterations"]
    assert np.abs(np.asarray(res["C"]) - np.asarray(r["C"])).max() <= 1e-12 * np.abs(r["C"]).max()
