"""Frozen weights of the ASG alpha selector (the reference's primary MLP, mlp_mse_20261031).

The reference loads ``exp/asg_independent_20261030/results/models/<name>/model.pt`` (a torch pickle of
a 92 -> 64 -> 32 -> 1 SiLU/sigmoid MLP with its input normalisation), after checking its sha256
against ``MODELS_FROZEN.json`` (``exp/asg_topopt_20261103/backend.py:95-100``). This package ships
the same numbers as a plain array file, ``asg_mlp_mse_20261031.npz``, converted once from that
checkpoint by

    python partial-green-jacobi_b200/asg_weights.py --ref <reference checkout>

which checks the checkpoint's sha256 against the frozen record first. ``load()`` checks the array
file against the sha256 recorded here, the same guard against a changed model.
"""
from __future__ import annotations

import argparse
import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
NAME = "mlp_mse_20261031"
WEIGHTS = HERE / f"asg_{NAME}.npz"
# sha256 of the source checkpoint (MODELS_FROZEN.json selected.mlp_mse.model_sha256)
SOURCE_SHA256 = "b48f57e82b1847be433df1a28e49f802f69ffbfe99336410b45f71216fb55289"
THRESHOLD = 0.2  # MODELS_FROZEN.json selected.mlp_mse.threshold: predictions below it select alpha = 0
ARRAYS = ("mean", "std", "mask", "w0", "b0", "w1", "b1", "w2", "b2")
# sha256 over the arrays above, float32 little-endian bytes in that order
ARRAYS_SHA256 = "7de767aad9c6c26101d2a8d56795b16bcd559aa7a81618d7a82c63c0fab62b6a"


def digest(arrays: dict) -> str:
    h = hashlib.sha256()
    for k in ARRAYS:
        h.update(np.ascontiguousarray(arrays[k], dtype="<f4").tobytes())
    return h.hexdigest()


def load(path: Path = WEIGHTS) -> dict:
    """The MLP's arrays (float32) and its threshold; raises if the file is not the frozen model."""
    with np.load(path) as z:
        arrays = {k: np.array(z[k], dtype=np.float32) for k in ARRAYS}
        source = str(z["source_sha256"])
    if source != SOURCE_SHA256 or (ARRAYS_SHA256 is not None and digest(arrays) != ARRAYS_SHA256):
        raise RuntimeError(f"{path.name} is not the frozen ASG model {NAME}")
    arrays["threshold"] = THRESHOLD
    return arrays


def convert(ref: Path, out: Path = WEIGHTS) -> str:
    """Checkpoint -> array file; returns the arrays' sha256 (the value of ARRAYS_SHA256)."""
    import torch

    results = ref / "exp/asg_independent_20261030/results"
    frozen = json.loads((results / "MODELS_FROZEN.json").read_text())
    selected = frozen["selected"][frozen["primary"]]
    if selected["name"] != NAME or selected["model_sha256"] != SOURCE_SHA256 or selected["threshold"] != THRESHOLD:
        raise RuntimeError(f"frozen selection changed: {selected}")
    ckpt = results / "models" / NAME / "model.pt"
    if hashlib.sha256(ckpt.read_bytes()).hexdigest() != SOURCE_SHA256:
        raise RuntimeError(f"{ckpt} does not match the frozen sha256")
    payload = torch.load(ckpt, map_location="cpu", weights_only=True)
    sd = payload["state_dict"]
    if payload["config"].get("inputs") != "full" or list(payload["config"]["widths"]) != [64, 32]:
        raise RuntimeError(f"unexpected model configuration {payload['config']}")
    arrays = {"mean": sd["mean"], "std": sd["std"], "mask": sd["mask"], "w0": sd["net.0.weight"],
              "b0": sd["net.0.bias"], "w1": sd["net.2.weight"], "b1": sd["net.2.bias"], "w2": sd["net.4.weight"],
              "b2": sd["net.4.bias"]}
    arrays = {k: v.numpy().astype(np.float32) for k, v in arrays.items()}
    np.savez(out, source_sha256=np.array(SOURCE_SHA256), **arrays)
    return digest(arrays)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", type=Path, required=True)
    print(convert(ap.parse_args().ref))
