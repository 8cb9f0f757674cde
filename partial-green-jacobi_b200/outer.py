"""Device-resident SIMP / OC outer loops over libpgj's filter, projection and OC kernels.

* ``ResidentOuter`` ~ ``exp/asg_gpu_resident_20261103/outer.py:12-59`` (Study I: periodic Gaussian,
  tanh projection at 1/2, SIMP eta=1e-4, 45 OC bisections).
* ``PaperOuter``    ~ ``exp/asg_sctop_reproduction_20261105/reproduction.py:69-118`` (Study II: clipped
  cone filter, tanh(beta, eta) projection, damped OC with the MATLAB bisection stop).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


def _sp():
    return _torch().cuda.current_stream().cuda_stream


def _p(t) -> int:
    return int(t.data_ptr())


def cone_stencil(rmin: float):
    """Offsets (dx, dy, dz) with weights rmin - |d| > 0, dz outer, then dx, then dy (reproduction.py:38-45)."""
    radius = math.ceil(rmin) - 1
    offsets, weights = [], []
    for dz in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            for dy in range(-radius, radius + 1):
                w = rmin - math.sqrt(dx * dx + dy * dy + dz * dz)
                if w > 0:
                    offsets.append([dx, dy, dz])
                    weights.append(w)
    return np.array(offsets, dtype=np.int32), np.array(weights)


def gaussian_weights(n: int):
    """Normalised Gaussian taps, sigma = 0.9 n / 32, radius int(4 sigma + 0.5) (outer.py:15-16)."""
    sigma = 0.9 * n / 32
    radius = int(4 * sigma + 0.5)
    q = np.arange(-radius, radius + 1, dtype=np.float64)
    w = np.exp(-0.5 * q * q / (sigma * sigma))
    return w / w.sum(), radius


class ResidentOuter:
    def __init__(self, n: int, volume: float = 0.3, move: float = 0.1):
        torch = _torch()
        self.n = n
        self.volume, self.move = volume, move
        w, self.radius = gaussian_weights(n)
        self.weights = torch.tensor(w, device="cuda", dtype=torch.float64)
        shape = (n, n, n)
        for name in ["x", "ph", "dp", "a", "energy", "new", "t"]:
            setattr(self, name, torch.empty(shape, device="cuda", dtype=torch.float64))
        self.scratch = torch.empty(4 * n ** 3 + 512, device="cuda", dtype=torch.float64)
        self.scratch[4 * n ** 3:4 * n ** 3 + 8].zero_()  # bisection bounds and the change record
        self.beta = 1.0

    @property
    def change(self):
        """max |new - x| of the last OC update: a (1,) device tensor, updated in place like the
        reference's ``outer.change`` (exp/asg_gpu_resident_20261103/outer.py:23,44)."""
        N = self.n ** 3
        return self.scratch[4 * N + 4:4 * N + 5]

    @property
    def bounds(self):
        """(lo, hi) of the last multiplier bisection, on the device (outer.py:22,38)."""
        N = self.n ** 3
        return self.scratch[4 * N:4 * N + 2]

    def capture(self):
        return None

    def set_initial(self, x):
        self.x.copy_(_torch().as_tensor(x, device="cuda", dtype=_torch().float64))

    def gaussian(self, x, out):
        L = _lib.lib()
        _lib.check(L.pgj_gaussian_filter(self.n, _p(self.weights), self.radius, _p(x.contiguous()), _p(out),
                                         _p(self.scratch), _sp()), "pgj_gaussian_filter")

    def evaluate(self, beta):
        self.beta = float(beta)
        self.gaussian(self.x, self.t)
        _lib.check(_lib.lib().pgj_study1_project(self.n, _p(self.t), self.beta, _p(self.ph), _p(self.dp), _p(self.a),
                                                 _sp()), "pgj_study1_project")

    def step(self, energy):
        self.energy.copy_(energy)
        ch = C.c_double()  # asking for the host copy makes the call return once the update is done
        _lib.check(_lib.lib().pgj_study1_oc(self.n, _p(self.weights), self.radius, _p(self.x), _p(self.ph),
                                            _p(self.dp), _p(self.energy), self.beta, self.volume, self.move,
                                            _p(self.new), _p(self.scratch), C.byref(ch), _sp()), "pgj_study1_oc")

    def advance(self):
        self.x.copy_(self.new)


class PaperOuter:
    def __init__(self, n, volume, rmin=3.0, beta=4.0, eta=0.5, emin=1e-9, move=0.1, exponent=0.3, floor=0.001):
        torch = _torch()
        self.n, self.volume, self.beta, self.eta, self.emin = n, volume, beta, eta, emin
        self.move, self.exponent, self.floor = move, exponent, floor
        offsets, weights = cone_stencil(rmin)
        self.offsets = torch.tensor(offsets, device="cuda")
        self.weights = torch.tensor(weights, device="cuda", dtype=torch.float64)
        for name in ["x", "ph", "dp", "a", "energy", "new", "t", "hs"]:
            setattr(self, name, torch.empty((n, n, n), device="cuda", dtype=torch.float64))
        self.scratch = torch.empty(4 * n ** 3 + 512, device="cuda", dtype=torch.float64)
        self.scratch[4 * n ** 3:4 * n ** 3 + 8].zero_()  # bisection bounds and the change record
        self.steps = 0
        self.raw_filter(torch.ones_like(self.x), self.hs)

    @property
    def change(self):
        """max |new - x| of the last OC update: a (1,) device tensor, updated in place (also by
        ``step_async``) like the reference's ``outer.change``."""
        N = self.n ** 3
        return self.scratch[4 * N + 4:4 * N + 5]

    @property
    def bounds(self):
        """(lo, hi, continue flag, bisection steps) of the last OC update on the device, the layout
        of the reference's ``outer.bounds`` (reproduction.py:77,96; outer.cu:34-38)."""
        N = self.n ** 3
        return self.scratch[4 * N:4 * N + 4]

    def raw_filter(self, x, out):
        _lib.check(_lib.lib().pgj_cone_filter(self.n, _p(self.offsets), _p(self.weights), self.weights.numel(),
                                              _p(x.contiguous()), _p(out), _sp()), "pgj_cone_filter")

    def capture(self):
        return None

    def set_initial(self, x):
        self.x.copy_(_torch().as_tensor(x, device="cuda", dtype=_torch().float64))

    def physical(self):
        self.raw_filter(self.x, self.t)
        _lib.check(_lib.lib().pgj_paper_project(self.n, _p(self.t), _p(self.hs), self.beta, self.eta, self.emin,
                                                _p(self.ph), _p(self.dp), _p(self.a), _sp()), "pgj_paper_project")

    def evaluate(self):
        self.physical()

    def step(self, e):
        self.energy.copy_(e)
        steps = C.c_int()
        ch = C.c_double()
        _lib.check(_lib.lib().pgj_paper_oc(self.n, _p(self.offsets), _p(self.weights), self.weights.numel(), _p(self.x),
                                           _p(self.ph), _p(self.dp), _p(self.hs), _p(self.energy), self.volume,
                                           self.beta, self.eta, self.emin, self.move, self.exponent, self.floor,
                                           _p(self.new), _p(self.scratch), C.byref(steps), C.byref(ch), _sp()),
                   "pgj_paper_oc")
        self.steps = steps.value

    def step_async(self, e):
        """OC update enqueued on the current stream without a host synchronisation; ``record()``
        reads (steps, change) afterwards from the device scratch."""
        if e.data_ptr() != self.energy.data_ptr():
            self.energy.copy_(e)
        _lib.check(_lib.lib().pgj_paper_oc(self.n, _p(self.offsets), _p(self.weights), self.weights.numel(), _p(self.x),
                                           _p(self.ph), _p(self.dp), _p(self.hs), _p(self.energy), self.volume,
                                           self.beta, self.eta, self.emin, self.move, self.exponent, self.floor,
                                           _p(self.new), _p(self.scratch), None, None, _sp()), "pgj_paper_oc")

    def record(self):
        """Device view of (steps, change) of the last asynchronous OC update."""
        N = self.n ** 3
        return self.scratch[4 * N + 3:4 * N + 5]

    def advance(self):
        self.x.copy_(self.new)
