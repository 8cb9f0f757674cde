"""Measurement tool: the Green apply on cuFFT (through torch.fft) timed beside libpgj's own passes.

    python partial-green-jacobi_b200/cufft_compare.py [--n 64] [--loads 6] [--reps 50]

Comparison only, never on the product path. The cuFFT form is the reference's Green apply
(exp/asg_gpu_resident_20261103/resident.py:104-117, spectral_three in scalar_fi.cu:38-44):
v = s (r - mean r); R2C over (z, y, x) of the three components of every load; the symmetric 3x3
symbol (1/N folded in); C2R with norm='forward'; z = s w - mean(s w). It is built from torch ops
(cuFFT plans, elementwise kernels) in FP64 and in FP32, with the symbol from pgj_green_symbol.
Against it: pgj_precondition (libpgj's standalone FP64 apply: five shared-memory FFT passes with the
symbol, scalings and projection fused) and, from pgj_profile_iteration, the transform kernels of
the slab-fused PCG iteration (which also carry the recurrence's vector updates). Prints one JSON line
with CUDA-event times (ms) and the relative difference of the two FP64 results.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--loads", type=int, default=6)
    ap.add_argument("--reps", type=int, default=50)
    args = ap.parse_args()
    import torch

    from __graft_entry__ import load_package

    pkg = load_package()
    n, L = args.n, args.loads
    ns = n // 2 + 1
    lam, mu = pkg.PAPER_MEDIUM
    a = torch.tensor(pkg.baseline_design(n, 0, 1e-6), device="cuda")
    op = pkg.Operator(n, L, lam, mu)
    op.set_material(a)
    op.set_alpha(0.5)
    s = op.scale.view(1, n, n, n, 3).permute(0, 4, 1, 2, 3).contiguous()  # (1, 3, n, n, n)
    sym = torch.empty((6, n, n, ns), dtype=torch.float64, device="cuda")
    pkg._lib.check(pkg._lib.lib().pgj_green_symbol(n, lam, mu, sym.data_ptr(),
                                                   torch.cuda.current_stream().cuda_stream), "pgj_green_symbol")
    g = torch.Generator(device="cuda").manual_seed(5)
    r = torch.randn((L, 3 * n ** 3), dtype=torch.float64, device="cuda", generator=g)

    def green_cufft(r, s, sym):
        rc = r.view(L, n, n, n, 3).permute(0, 4, 1, 2, 3)              # (L, 3, n, n, n)
        v = s * (rc - rc.mean(dim=(2, 3, 4), keepdim=True))
        V = torch.fft.rfftn(v, dim=(2, 3, 4))
        x, y, zc = V[:, 0], V[:, 1], V[:, 2]
        c0, c1, c2, c3, c4, c5 = sym
        W = torch.stack((c0 * x + c3 * y + c4 * zc, c3 * x + c1 * y + c5 * zc, c4 * x + c5 * y + c2 * zc), dim=1)
        w = torch.fft.irfftn(W, s=(n, n, n), dim=(2, 3, 4), norm="forward")
        sw = s * w
        z = sw - sw.mean(dim=(2, 3, 4), keepdim=True)
        return z.permute(0, 2, 3, 4, 1).reshape(L, -1)

    def timed(fn, reps):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"n": n, "loads": L, "reps": args.reps}
    z_ref = green_cufft(r, s, sym)
    z_pgj = op.apply_precond(r)
    torch.cuda.synchronize()
    out["fp64_rel_diff"] = float((z_pgj - z_ref).abs().max() / z_ref.abs().max())
    out["cufft_fp64_ms"] = timed(lambda: green_cufft(r, s, sym), args.reps)
    out["pgj_precondition_fp64_ms"] = timed(lambda: op.apply_precond(r), args.reps)
    r32, s32, sym32 = r.float(), s.float(), sym.float()
    out["cufft_fp32_ms"] = timed(lambda: green_cufft(r32, s32, sym32), args.reps)
    # the cuFFT transforms alone (R2C + C2R of the 3L fields), without the torch elementwise work
    v = r.view(L, n, n, n, 3).permute(0, 4, 1, 2, 3).contiguous()
    V = torch.fft.rfftn(v, dim=(2, 3, 4))
    out["cufft_transforms_only_fp64_ms"] = timed(
        lambda: torch.fft.irfftn(torch.fft.rfftn(v, dim=(2, 3, 4)), s=(n, n, n), dim=(2, 3, 4), norm="forward"),
        args.reps)
    v32 = v.float()
    out["cufft_transforms_only_fp32_ms"] = timed(
        lambda: torch.fft.irfftn(torch.fft.rfftn(v32, dim=(2, 3, 4)), s=(n, n, n), dim=(2, 3, 4), norm="forward"),
        args.reps)
    del V
    for prec in ("fp64", "mixed"):
        o = pkg.Operator(n, L, lam, mu, precision=prec)
        o.set_material(a)
        o.set_alpha(0.5)
        prof = o.profile_iteration(np.eye(6)[:L] if L <= 6 else np.tile(np.eye(6), (L // 6 + 1, 1))[:L], reps=20)
        out[f"pgj_fused_transform_kernels_{prec}_ms"] = {k: v["ms"] for k, v in prof.items() if k != "operator"}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
