"""Global alpha selectors of the density-selector study: small reductions over the density field that
pick the one exponent alpha of the partial Green-Jacobi scaling D^{-alpha/2} for a design.

They follow ``exp/asg_density_selector_20261105/run.py:27-43,53-67`` (contrast, gray, compact8 and
compact8q; the frozen parameters of ``MODELS_FROZEN.json``), the compact-law features of
``solver/experiments/global_alpha_compact_law/law.py:10-19`` and the ASG MLP
(``exp/asg_gpu_resident_20261103/resident.py:160-162``: the 92 full-grid statistics of
``solver/experiments/global_alpha_stats/features.py:17-49`` through the frozen network of
``solver/experiments/asg_independent/train.py:27-35``, weights in ``asg_weights``). Each returns a 0-d float64 tensor on
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


# ASG features: CDF points of q, shifts of the periodic differences (in cells: 1, 2, n/16, n/8)
ASG_CDF = (0.01, 0.05, 0.25, 0.5, 0.75, 0.95, 0.99)


def asg_features(a):
    """The 92 statistics of the log density rescaled to q in [0, 1], in FP32 like the reference:
    mean and variance of q, 7 CDF values; per axis (z, y, x) and shift (1, 2, n/16, n/8 cells) of the
    periodic difference d: mean |d|, mean d^2, mean d^4, max |d|, fraction |d| > 1e-6, fraction
    |d| > 0.25; per axis the scaling exponent log2(s2(2) / s2(1)) and the jump ratio s2 / s1 at
    shift 1; the three normalised cross-correlations of the unit-shift differences; the log contrast
    over log 1e4 and 1 / n. Needs n >= 32 and n a multiple of 16 (the reference asserts the same)."""
    torch = _torch()
    ell = a.float().log()
    lo, hi = torch.aminmax(ell)
    span = hi - lo
    q = (ell - lo) / span.clamp_min(1e-12)
    n = q.shape[0]
    if q.shape != (n, n, n) or n < 32 or n % 16:
        raise ValueError("the ASG features need a cubic grid with n >= 32 and n a multiple of 16")
    mean = q.mean()
    values = [mean, (q - mean).square().mean()]
    values += [(q <= t).float().mean() for t in ASG_CDF]
    pairs, unit = [], []
    for axis in range(3):
        sums = []
        for shift in (1, 2, max(1, n // 16), max(1, n // 8)):
            diff = torch.roll(q, -shift, axis) - q
            d = diff.abs()
            s1, s2 = d.mean(), d.square().mean()
            values += [s1, s2, d.square().square().mean(), d.amax(), (d > 1e-6).float().mean(),
                       (d > 0.25).float().mean()]
            sums.append((s1, s2))
            if shift == 1:
                unit.append(diff)
        s1, s2 = sums[0]
        exponent = torch.where(s2 > 1e-20, (sums[1][1] / s2.clamp_min(1e-20)).clamp_min(1e-20).log2(),
                               torch.zeros_like(s2))
        pairs += [exponent, s2 / s1.clamp_min(1e-20)]
    values += pairs
    norm = (unit[0].square().mean() + unit[1].square().mean() + unit[2].square().mean()).clamp_min(1e-20)
    values += [(unit[0] * unit[1]).mean() / norm, (unit[0] * unit[2]).mean() / norm,
               (unit[1] * unit[2]).mean() / norm, span / math.log(10000.0), q.new_tensor(1.0 / n)]
    return torch.stack(values)


_ASG_NET = {}


def _asg_net(device):
    """The frozen MLP's tensors on `device` (loaded and checked once per device)."""
    torch = _torch()
    key = str(device)
    if key not in _ASG_NET:
        from . import asg_weights

        w = asg_weights.load()
        _ASG_NET[key] = {k: (torch.tensor(v, device=device) if k != "threshold" else v) for k, v in w.items()}
    return _ASG_NET[key]


def asg_prediction(a):
    """Raw MLP output in (0, 1): sigmoid(L2 silu(L1 silu(L0 ((x - mean) / std * mask)))), FP32."""
    torch = _torch()
    net = _asg_net(a.device)
    x = (asg_features(a) - net["mean"]) / net["std"] * net["mask"]
    h = torch.nn.functional.silu(net["w0"] @ x + net["b0"])
    h = torch.nn.functional.silu(net["w1"] @ h + net["b1"])
    return torch.sigmoid(net["w2"] @ h + net["b2"]).reshape(())


def asg_alpha(a):
    """ASG alpha: the MLP prediction, or 0 (the plain Green preconditioner) below the frozen
    threshold 0.2 (resident.py:160-162); a 0-d float64 tensor on the input's device."""
    torch = _torch()
    pred = asg_prediction(a)
    return torch.where(pred < _asg_net(a.device)["threshold"], torch.zeros_like(pred), pred).double()


def _torch():
    import torch

    return torch
