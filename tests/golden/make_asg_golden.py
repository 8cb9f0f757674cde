"""Golden vectors of the ASG alpha selector from the reference's own code, run here on CPU.

    python tests/golden/make_asg_golden.py [--ref /root/reference]

For seeded density multipliers (SIMP of the benchmark generator, n in {32, 48, 64}, Emin in
{1e-4, 1e-6, 1e-9}) it evaluates the reference's feature extractor
(solver/experiments/global_alpha_stats/features.py `extract`) and its frozen primary network (the
`Model` class of solver/experiments/asg_independent/train.py, loaded from the checkpoint named in
exp/asg_independent_20261030/results/MODELS_FROZEN.json after the sha256 check), and writes the
fields' seeds, the 92 features and the raw predictions to tests/golden/asg_selector.npz.
"""
from __future__ import annotations

import argparse
import ast
import hashlib
import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
CASES = [(32, 0, 1e-4), (32, 1, 1e-9), (48, 2, 1e-6), (64, 3, 1e-6), (64, 4, 1e-9), (32, 5, 1e-6)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ref = Path(ap.parse_args().ref)
    import torch
    from torch import nn

    spec = importlib.util.spec_from_file_location("ref_features", ref / "solver/experiments/global_alpha_stats/features.py")
    feats = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(feats)
    # the reference Model class, extracted by name from its training script (as its backend does)
    tree = ast.parse((ref / "solver/experiments/asg_independent/train.py").read_text())
    node = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == "Model")
    ns = {"nn": nn, "torch": torch}
    exec(compile(ast.Module(body=[node], type_ignores=[]), "train.py", "exec"), ns)
    results = ref / "exp/asg_independent_20261030/results"
    frozen = json.loads((results / "MODELS_FROZEN.json").read_text())
    sel = frozen["selected"][frozen["primary"]]
    ckpt = results / "models" / sel["name"] / "model.pt"
    assert hashlib.sha256(ckpt.read_bytes()).hexdigest() == sel["model_sha256"]
    payload = torch.load(ckpt, map_location="cpu", weights_only=True)
    net = ns["Model"](payload["config"])
    net.load_state_dict(payload["state_dict"])
    net.eval()
    sys.path.insert(0, str(REPO / "oracle"))
    import pgj_oracle as O

    features, preds = [], []
    for n, seed, emin in CASES:
        a = torch.tensor(O.simp(O.baseline_density(n, seed), emin))
        with torch.no_grad():
            f = feats.extract(a)
            p = net(f)
        features.append(f.reshape(-1).numpy())
        preds.append(float(p.reshape(())))
    np.savez(HERE / "asg_selector.npz", cases=np.array(CASES), features=np.array(features, dtype=np.float32),
             predictions=np.array(preds, dtype=np.float64), threshold=np.array(sel["threshold"]))
    print(preds)


if __name__ == "__main__":
    main()
