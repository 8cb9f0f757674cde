"""Generate tests/golden/selector_law.npz: the compact-law features and law8 values of the reference.

Run in a container that has the reference tree (default /root/reference) and a CPU torch:

    python tests/golden/make_selector_golden.py [--ref /root/reference]

It imports the reference's ``solver/experiments/global_alpha_compact_law/law.py`` (plain torch,
CPU-runnable) and evaluates ``extract_law`` and ``evaluate(..., CONFIGS['law8'])`` on seeded
density fields: SIMP designs of the benchmark generator at three weak-material ratios and three
grid sizes, a homogeneous field and a two-phase layered field. The fields and the outputs are
written together; nothing at test time reads the reference tree.
"""
from __future__ import annotations

import argparse
import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def fields():
    sys.path.insert(0, str(REPO / "oracle"))
    import pgj_oracle as oracle

    out = {}
    for k, (n, emin, seed) in enumerate([(8, 1e-4, 0), (10, 1e-6, 1), (12, 1e-9, 2), (12, 1e-6, 3), (10, 1e-4, 4)]):
        out[f"simp{k}"] = oracle.simp(oracle.baseline_density(n, seed), emin)
    out["homogeneous"] = np.full((8, 8, 8), 0.37)
    layered = np.full((8, 8, 8), 1e-6)
    layered[:, :, :3] = 1.0
    out["layered"] = layered
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ref = Path(ap.parse_args().ref)
    import torch

    spec = importlib.util.spec_from_file_location("law", ref / "solver/experiments/global_alpha_compact_law/law.py")
    law = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(law)
    save = {}
    for name, a in fields().items():
        f = law.extract_law(torch.tensor(a, dtype=torch.float64))
        save[f"{name}/a"] = a
        save[f"{name}/features"] = f.numpy().astype(np.float32)
        save[f"{name}/law8"] = np.float64(law.evaluate(f, law.CONFIGS["law8"]))
    np.savez_compressed(HERE / "selector_law.npz", **save)
    print("wrote", HERE / "selector_law.npz", len(save), "arrays")


if __name__ == "__main__":
    main()
