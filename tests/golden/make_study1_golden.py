"""Extract the archived full Study I trajectories (180-step shear design, alpha 0.5) from the
reference checkout into tests/golden/study1_full.json.

    python tests/golden/make_study1_golden.py [--ref /root/reference]

Source: data/study1/full_timing.csv (one row per grid, seed and load mode; written by the
reference's exp/asg_scaling_20261104/study.py `full`): the final objective J (mean of the three
shear moduli), the final volume, the number of design steps taken and the stop-rule flag. Nothing
here runs on the GPU; the tests only read the JSON.
"""
from __future__ import annotations

import argparse
import csv
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    src = Path(ap.parse_args().ref) / "data/study1/full_timing.csv"
    rows = []
    with src.open() as fh:
        for r in csv.DictReader(fh):
            rows.append(dict(n=int(r["n"]), seed=int(r["seed"]), load_mode=r["load_mode"], steps=int(r["steps"]),
                             optimization_converged=r["optimization_converged"] == "True", J=float(r["J"]),
                             volume=float(r["volume"]), mean_step_ms=float(r["mean_step_ms"])))
    (HERE / "study1_full.json").write_text(json.dumps(dict(source="data/study1/full_timing.csv", method="0.5",
                                                           rows=rows), indent=1) + "\n")
    print(f"wrote {len(rows)} rows")


if __name__ == "__main__":
    main()
