"""Generate the FP64 drop-in parity fixtures of the benchmark grid from the CPU oracle.

    python tests/golden/make_config2.py [--workers 7] [--set all|n32|n64]

Each case is one certified six-load homogenization of a seeded synthetic design (N(0,1) noise,
periodic Gaussian sigma = n/16, logistic threshold to volume fraction 0.35, SIMP p = 3 with
E0 = 1, nu = 0.3), zero start, relative true residual 1e-8, solved by the oracle twice: in its
default summation order ("a") and in a second order ("b": recurrence dots and operator corner
sums reordered), and for some cases a third time with the operator evaluated by the reference's own
modal element arithmetic ("r", fi_modal.cuh compiled on the host by oracle/Makefile). The fixture
keeps C_H, the per-load iteration counts of every order, the relative true residuals and the rhs
norms. The spread between the orders shows how far the counts move with rounding alone; the GPU
tests' count tolerances are stated against it.

Grids: n = 32, alpha in {0, 0.5, 1} x Emin/E0 in {1e-4, 1e-6, 1e-9} x seeds 0..4 (45 cases),
n = 64, alpha = 0.5 x Emin/E0 in {1e-4, 1e-6, 1e-9}, seed 0 (3 cases), and one high-contrast case
that reaches the iteration cap, n = 54, alpha 0.5, Emin/E0 1e-9, seed 0 (``--set all``, written to
config2.json). ``--set config3 --orders a --out tests/golden/config3.json`` writes the mixed-precision
grids' FP64 references: n = 96 at Emin/E0 1e-6 and 1e-9 and n = 128 at 1e-6, alpha 0.5, seed 0
(hours of host time each). The n = 64 cases take
about an hour of single-core time each, so the script runs a spawn-started process pool and
checkpoints finished runs to ``--checkpoint`` so that an interrupted run resumes.
Nothing here runs on the GPU or reads the reference tree.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]

ALPHAS = (0.0, 0.5, 1.0)
EMINS = (1e-4, 1e-6, 1e-9)


def cases(which: str):
    out = []
    if which in ("all", "n64"):
        for emin in EMINS:
            out.append((64, 0.5, emin, 0))
    if which in ("all", "cap"):
        # high contrast at alpha 0.5: the device FP64 recurrence reaches the 4000-iteration cap here;
        # the oracle decides whether the reference would too
        out.append((54, 0.5, 1e-9, 0))
    if which == "config3":
        # the mixed-precision grids: the FP64 oracle's C_H is what the mixed results are held to
        out += [(96, 0.5, 1e-6, 0), (96, 0.5, 1e-9, 0), (128, 0.5, 1e-6, 0)]
    if which in ("all", "n32"):
        for alpha in ALPHAS:
            for emin in EMINS:
                for seed in range(5):
                    out.append((32, alpha, emin, seed))
    return out


def key(case) -> str:
    n, alpha, emin, seed = case
    return f"n{n}/a{alpha:g}/e{emin:g}/s{seed}"


def run_one(args):
    case, order = args
    os.environ.setdefault("PGJ_ORACLE_THREADS", "1")
    sys.path.insert(0, str(REPO / "oracle"))
    import numpy as np
    import pgj_oracle as o

    n, alpha, emin, seed = case
    a = o.simp(o.baseline_density(n, seed), emin)
    t0 = time.time()
    res = o.homogenize(a, *o.PAPER, alpha, rtol=1e-8, order=order)
    rec = dict(key=key(case), order=order, n=n, alpha=alpha, emin=emin, seed=seed,
               iterations=[i.iterations for i in res["infos"]],
               relative_residual=[i.relative_residual for i in res["infos"]],
               rhs_norm=[i.rhs_norm for i in res["infos"]],
               converged=[i.converged for i in res["infos"]],
               restarts=res["infos"][0].restarts, raised=bool(res["raised"]),
               C=np.asarray(res["C"]).tolist(), seconds=time.time() - t0)
    return rec


def merge(records: list[dict]) -> dict:
    by = {}
    for r in records:
        by.setdefault(r["key"], {})[r["order"]] = r
    out = {}
    for k, d in sorted(by.items()):
        if "a" not in d:
            continue
        a = d["a"]
        b = d.get("b")
        r = d.get("r")
        out[k] = dict(n=a["n"], alpha=a["alpha"], emin=a["emin"], seed=a["seed"], C=a["C"],
                      iterations=a["iterations"],
                      iterations_b=b["iterations"] if b else None,
                      C_b=b["C"] if b else None,
                      iterations_r=r["iterations"] if r else None,
                      relative_residual=a["relative_residual"], rhs_norm=a["rhs_norm"],
                      converged=a["converged"], restarts=a["restarts"], raised=a["raised"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--set", default="all", choices=("all", "n32", "n64", "cap", "config3"))
    ap.add_argument("--checkpoint", default="/tmp/pgj_config2_checkpoint.jsonl")
    ap.add_argument("--out", default=str(HERE / "config2.json"))
    ap.add_argument("--merge-only", action="store_true", help="write the fixture from the checkpoint, run nothing")
    ap.add_argument("--orders", default="ab", help="a: default, b: reordered sums, r: the reference's modal "
                                                   "element arithmetic (needs oracle/_ref, built by oracle/Makefile)")
    args = ap.parse_args()

    ckpt = Path(args.checkpoint)
    done = []
    if ckpt.exists():
        done = [json.loads(line) for line in ckpt.read_text().splitlines() if line.strip()]
    have = {(r["key"], r["order"]) for r in done}
    todo = [(c, o) for c in cases(args.set) for o in args.orders if (key(c), o) not in have]
    print(f"{len(done)} runs checkpointed, {len(todo)} to go", flush=True)

    import multiprocessing as mp

    if todo and not args.merge_only:
        with mp.get_context("spawn").Pool(args.workers) as pool, ckpt.open("a") as fh:
            for rec in pool.imap_unordered(run_one, todo):
                fh.write(json.dumps(rec) + "\n")
                fh.flush()
                done.append(rec)
                print(f"{rec['key']} {rec['order']}: its {rec['iterations']} in {rec['seconds']:.0f} s",
                      flush=True)

    merged = merge(done)
    Path(args.out).write_text(json.dumps(dict(
        source=f"tests/golden/make_config2.py --set {args.set} (CPU oracle, orders {args.orders})",
        physics=dict(E0=1.0, nu=0.3, p=3, vf=0.35, sigma="n/16", width=0.1, rtol=1e-8),
        cases=merged), indent=1) + "\n")
    print(f"wrote {len(merged)} cases to {args.out}")


if __name__ == "__main__":
    main()
