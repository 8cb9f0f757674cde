#!/usr/bin/env python
"""Per-kernel CUDA-event timing of one PCG iteration (the kernels a certified solve loops over).

    python partial-green-jacobi_b200/profile_iteration.py --n 64 --precision mixed --reps 20

Builds a context for the seeded baseline design (n, Emin=1e-6, alpha=0.5, paper medium), runs the
certification and first direction, then times `reps` iterations kernel by kernel through
pgj_profile_iteration (the same kernels the solve graphs launch, issued directly so that a profiler
sees each launch). Prints the tile shapes, the iteration time and per-kernel times with the
algorithmic bytes per second. Tile autotuners can be pinned with PGJ_STENCIL_TY / PGJ_STENCIL_ZC /
PGJ_FFT_RB / PGJ_FFT_NKY / PGJ_FFT_NKZ.
"""
import argparse
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--emin", type=float, default=1e-6)
    ap.add_argument("--unfused", action="store_true", help="time the step-by-step kernel set")
    args = ap.parse_args()
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    op = pkg.Operator(args.n, 6, *pkg.PAPER_MEDIUM, precision=args.precision)
    if args.unfused:
        op.set_fused_iteration(False)
    op.set_material(torch.tensor(pkg.baseline_design(args.n, 0, args.emin), device="cuda"))
    op.set_alpha(0.5)
    prof = op.profile_iteration(np.eye(6), reps=args.reps)
    torch.cuda.synchronize()
    tot = sum(v["ms"] for v in prof.values())
    print(f"n={args.n} precision={args.precision} tiles={op.tile_shapes()} iteration {tot * 1e3:.1f} us")
    for k, v in prof.items():
        print(f"  {k:18s} {v['ms'] * 1e3:8.1f} us  {v['bytes'] / v['ms'] / 1e6:8.1f} GB/s")


if __name__ == "__main__":
    main()
