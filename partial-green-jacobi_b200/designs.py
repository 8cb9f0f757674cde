"""Seeded synthetic design fields (host-side input generation; not on the device hot path).

``baseline_density``: N(0,1) noise -> periodic Gaussian filter (sigma = n/16 cells) -> smooth
threshold at the (1 - vf) quantile, rho = logistic((f - q_{1-vf}) / (width * std f)), width 0.1.
``simp``: E = Emin + rho^p (E0 - Emin), E0 = 1, p = 3.
``uneven_designs``: the batched uneven-design workload, one seeded (n, volume fraction, alpha)
draw per design with n from {24, 32, 48, 64}, vf uniform in [0.2, 0.5] and alpha uniform in [0, 1].
``study1_initial`` / ``study1_state0``: the reference's Study I initial design and its state 0,
material(physical(initial(n, seed), 1)[0]) (exp/asg_topopt_20261103/study.py:61-88).
"""
from __future__ import annotations

import numpy as np


def baseline_density(n: int, seed: int, vf: float = 0.35, sigma_cells: float | None = None,
                     width: float = 0.1) -> np.ndarray:
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n, n, n))
    f = gaussian_filter(noise, n / 16.0 if sigma_cells is None else sigma_cells, mode="wrap")
    q = np.quantile(f, 1.0 - vf)
    return 1.0 / (1.0 + np.exp(-(f - q) / (width * f.std())))


def simp(rho: np.ndarray, emin: float, p: float = 3.0) -> np.ndarray:
    return emin + rho ** p * (1.0 - emin)


def baseline_design(n: int, seed: int, emin: float, vf: float = 0.35) -> np.ndarray:
    return simp(baseline_density(n, seed, vf), emin)


UNEVEN_GRIDS = (24, 32, 48, 64)


def uneven_spec(seed: int) -> tuple[int, float, float]:
    """(n, volume fraction, alpha) of design `seed` of the uneven batch (its own generator stream)."""
    rng = np.random.default_rng([seed, 4])
    n = int(rng.choice(UNEVEN_GRIDS))
    vf = float(rng.uniform(0.2, 0.5))
    alpha = float(rng.uniform(0.0, 1.0))
    return n, vf, alpha


def uneven_designs(count: int = 64, emin: float = 1e-6):
    """Designs 0..count-1 of the uneven batch: [(seed, n, vf, alpha, a)], a = SIMP(baseline density)."""
    out = []
    for seed in range(count):
        n, vf, alpha = uneven_spec(seed)
        out.append((seed, n, vf, alpha, baseline_design(n, seed, emin, vf)))
    return out


def _study1_physical(x, beta):
    from scipy.ndimage import gaussian_filter

    t = gaussian_filter(x, 0.9 * x.shape[0] / 32, mode="wrap")
    den = 2 * np.tanh(beta / 2)
    return (np.tanh(beta / 2) + np.tanh(beta * (t - 0.5))) / den


def study1_initial(n: int, seed: int = 20261104) -> np.ndarray:
    """Study I initial design density: 12 random periodic cosine modes (std 0.12) around 0.3,
    shifted by 50 bisections so that the beta = 1 physical density has volume 0.3
    (exp/asg_topopt_20261103/study.py:75-88)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*([(np.arange(n) + 0.5) / n] * 3), indexing="ij")
    field = np.zeros((n, n, n))
    for _ in range(12):
        k = rng.integers(-2, 3, 3)
        if not np.any(k):
            k[0] = 1
        field += rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + rng.uniform(0, 2 * np.pi))
    field = 0.12 * field / field.std()
    lo, hi = -1.0, 1.0
    cand = None
    for _ in range(50):
        shift = (lo + hi) / 2
        cand = np.clip(0.3 + field + shift, 0.01, 0.99)
        if _study1_physical(cand, 1.0).mean() > 0.3:
            hi = shift
        else:
            lo = shift
    return cand


def study1_state0(n: int, seed: int = 20261104) -> np.ndarray:
    ph = _study1_physical(study1_initial(n, seed), 1.0)
    return 1e-4 + (1 - 1e-4) * ph ** 3
