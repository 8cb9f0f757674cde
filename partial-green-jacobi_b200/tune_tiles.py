#!/usr/bin/env python
"""The tile tuner: times every candidate tile shape of the operator and the Green passes on this GPU
and writes the table libpgj builds in (csrc/pgj_tiles.inc).

    python partial-green-jacobi_b200/tune_tiles.py [--sizes 16,24,32] [--out csrc/pgj_tiles.inc]

For every grid edge (default: all supported even 5-smooth n from 4 to 128) and both precisions it
creates a six-load context with PGJ_AUTOTUNE=1, so that the context's creation times the candidates
(operator rows / z-planes / plane buffers / occupancy variant; FFT rows per x block, y and z chunks)
instead of reading the table, and records the fastest. With the table built in, contexts take their
shapes without timing anything: the block decomposition, and so the summation order of every block
partial sum, is the same in every process and batch. Rebuild libpgj after writing the table.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))


def supported(n: int) -> bool:
    if n < 4 or n % 2:
        return False
    m = n
    for r in (2, 3, 5):
        while m % r == 0:
            m //= r
    return m == 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="")
    ap.add_argument("--max-n", type=int, default=128)
    ap.add_argument("--out", type=Path, default=HERE / "csrc" / "pgj_tiles.inc")
    args = ap.parse_args()
    os.environ["PGJ_AUTOTUNE"] = "1"
    import torch

    from __graft_entry__ import load_package

    pkg = load_package()
    sizes = [int(s) for s in args.sizes.split(",") if s] or [n for n in range(4, args.max_n + 1) if supported(n)]
    rows = []
    for n in sizes:
        for prec, code in (("fp64", 0), ("mixed", 1)):
            op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM, precision=prec)
            cfg = (C.c_int * 9)()
            pkg._lib.check(pkg._lib.lib().pgj_tile_config(op._ctx, cfg), "pgj_tile_config")
            rows.append((n, code, cfg[0], cfg[1], cfg[2], cfg[3], cfg[4], cfg[5], cfg[6]))
            print(f"n={n} {prec}: {rows[-1]}", flush=True)
            del op
            torch.cuda.empty_cache()
    gpu = torch.cuda.get_device_name()
    lines = ["// Tile shapes per (grid edge, precision): n, precision (0 FP64, 1 FP32), operator rows per block,",
             "// operator z-planes per block, plane buffers, occupancy variant, FFT rows per x block, y chunks, z chunks.",
             f"// Written by partial-green-jacobi_b200/tune_tiles.py from timings on one {gpu}."]
    lines += ["    {" + ", ".join(str(v) for v in r) + "}," for r in rows]
    args.out.write_text("\n".join(lines) + "\n")
    print(f"wrote {len(rows)} entries to {args.out}")


if __name__ == "__main__":
    main()
