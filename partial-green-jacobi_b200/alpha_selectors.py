"""Global alpha selectors of the density-selector study: small reductions over the density field that
pick the one exponent alpha of the partial Green-Jacobi scaling D^{-alpha/2} for a design.

They follow ``exp/asg_density_selector_20261105/run.py:27-43,53-67`` (contrast, gray, compact8 and
compact8q; the frozen parameters of ``MODELS_FROZEN.json``) and the compact-law features of
``solver/experiments/global_alpha_compact_law/law.py:10-19``. Each returns a 0-d float64 tensor on
the input's device. They are device-agnostic torch reductions over N values (one scalar per design
step, off the PCG path), run on the design's own device without a host round trip.
"""
from __future__ import annotations

import math

# frozen selector parameters (MODELS_FROZEN.json models.*.anchors, models.gray.gamma / g_ref)
CONTRAST_ANCHORS = (0.5625, 0.6875, 0.8125)
GRAY_ANCHORS = (0.5625, 0.75, 0.8125)
GRAY_GAMMA = 0.075
GRAY_G_REF = 0.3739899920170806
# compact law with exponent 8 (law.py CONFIGS['law8']) and the selector's cut-off below which
# alpha is 0 (the plain Green preconditioner)
COMPACT_COEFFICIENT = 0.75
COMPACT_THRESHOLD = 2.5
COMPACT_EXPONENT = 8
COMPACT_CUTOFF = 0.375


def _contrast_base(a, anchors):
    """Piecewise-linear alpha over the decades of contrast s = log10(max a / min a) in [0, 9]."""
    torch = _torch()
    lo, hi = torch.aminmax(a)
    s = torch.log10(hi / lo).clamp(0.0, 9.0)
    b4, b6, b9 = anchors
    base = torch.where(s < 4, b4 * s / 4, torch.where(s < 6, b4 + (b6 - b4) * (s - 4) / 2, b6 + (b9 - b6) * (s - 6) / 3))
    return s, base


def _quantize16(value, s):
    torch = _torch()
    return torch.where(s > 1e-12, (value.clamp(0, 1) * 16 + 0.5).floor() / 16, torch.zeros_like(value))


def contrast_alpha(a, anchors=CONTRAST_ANCHORS):
    """alpha from the material contrast alone, rounded to sixteenths (run.py:27-33)."""
    s, base = _contrast_base(a.double(), anchors)
    return _quantize16(base, s)


def gray_alpha(a, rho, anchors=GRAY_ANCHORS, gamma=GRAY_GAMMA, g_ref=GRAY_G_REF):
    """Contrast alpha shifted by the grayness g = (v - mean rho^2) / (v (1 - v)), v = mean rho,
    of the physical density rho (run.py:36-43)."""
    s, base = _contrast_base(a.double(), anchors)
    rho = rho.double()
    v = rho.mean()
    g = ((v - rho.square().mean()) / (v * (1 - v) + 1e-12)).clamp(0, 1)
    return _quantize16(base + gamma * (g_ref - g), s)


def law_features(a):
    """(area, jump, contrast, complexity) of law.py:10-19, in FP32 like the reference.

    q is log a rescaled to [0, 1]; per axis the periodic forward differences d give mean |d|,
    mean d^2 and the fraction of |d| > 1e-6. area = mean active fraction, jump = sum mean d^2 /
    sum mean |d|, contrast = log(max a / min a) / log(1e4), complexity = area * n.
    """
    torch = _torch()
    ell = a.float().log()
    lo, hi = torch.aminmax(ell)
    span = hi - lo
    q = (ell - lo) / span.clamp_min(1e-12)
    n = q.shape[0]
    s1, s2, active = [], [], []
    for axis in range(3):
        d = (torch.roll(q, -1, axis) - q).abs()
        s1.append(d.mean())
        s2.append(d.square().mean())
        active.append((d > 1e-6).float().mean())
    total1 = s1[0] + s1[1] + s1[2]
    total2 = s2[0] + s2[1] + s2[2]
    area = (active[0] + active[1] + active[2]) / 3
    jump = total2 / total1.clamp_min(1e-20)
    return torch.stack((area, jump, span / math.log(10000.0), area * n))


def compact8_alpha(a, quantize=False):
    """alpha = 1 - 0.75 sqrt(area jump / contrast) - (2.5 / complexity)^8, clamped to [0, 1], 0 for
    a homogeneous field and below 0.375; ``quantize`` rounds to sixteenths (compact8q)
    (run.py:60-66)."""
    torch = _torch()
    area, jump, contrast, complexity = law_features(a).to(torch.float64).unbind()
    value = (1.0 - COMPACT_COEFFICIENT * (area * jump).clamp_min(0).sqrt() / contrast.clamp_min(1e-30).sqrt()
             - (COMPACT_THRESHOLD / complexity.clamp_min(1e-30)) ** COMPACT_EXPONENT)
    value = torch.where((complexity > 1e-12) & (contrast > 1e-12), value.clamp(0.0, 1.0), torch.zeros_like(value))
    value = torch.where(value < COMPACT_CUTOFF, torch.zeros_like(value), value)
    if quantize:
        value = (16 * value + 0.5).floor() / 16
    return value


def _torch():
    import torch

    return torch
