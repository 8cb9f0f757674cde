"""Concurrent certified homogenizations of many independent designs on one GPU.

Every kernel of one homogenization is latency-bound at n <= 64 (a few waves of small blocks), so one
design cannot fill a B200. ``Batch`` keeps ``slots`` libpgj contexts per grid size, each on its own
CUDA stream, and enqueues whole certified solves with ``pgj_solve_async`` (one graph launch per
design: restarts, PCG loop and certification are decided on the device). Designs of different n
run side by side; results are collected with one synchronisation per design. This is the batched
form of the reference's per-design loop (``exp/asg_density_selector_20261105/run.py:105-119``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .resident import PAPER_MEDIUM, Operator


def _torch():
    import torch

    return torch


@dataclass
class Request:
    """One homogenization: density multiplier a (n^3), preconditioner exponent alpha."""
    a: object
    alpha: float
    tag: object = None


@dataclass
class Result:
    tag: object
    C: np.ndarray
    infos: list
    status: int
    refinements: int
    launches: int
    latency_ms: float  # device time from the request's first copy to its C_H on the slot's stream


@dataclass
class _Slot:
    op: Operator
    stream: object
    u: object
    C: object
    Ch: object
    event: object = None
    start: object = None
    req: Request | None = None
    a_dev: object = None


class Batch:
    def __init__(self, slots: int = 4, precision: str = "mixed", medium=PAPER_MEDIUM, rtol: float = 1e-8,
                 macros=None):
        self.slots = int(slots)
        self.precision = precision
        self.lam, self.mu = medium
        self.rtol = float(rtol)
        self.macros = np.ascontiguousarray(np.eye(6) if macros is None else np.atleast_2d(macros), dtype=np.float64)
        self.pool: dict[int, list[_Slot]] = {}

    def _slots_for(self, n: int) -> list[_Slot]:
        torch = _torch()
        if n not in self.pool:
            slots = []
            for _ in range(self.slots):
                stream = torch.cuda.Stream()
                with torch.cuda.stream(stream):
                    op = Operator(n, self.macros.shape[0], self.lam, self.mu, self.precision)
                    u = torch.zeros((self.macros.shape[0], 3 * n ** 3), dtype=torch.float64, device="cuda")
                    Cd = torch.empty((6, 6), dtype=torch.float64, device="cuda")
                    Ch = torch.empty((6, 6), dtype=torch.float64).pin_memory()
                slots.append(_Slot(op, stream, u, Cd, Ch))
            torch.cuda.synchronize()
            self.pool[n] = slots
        return self.pool[n]

    def _launch(self, slot: _Slot, req: Request) -> None:
        torch = _torch()
        with torch.cuda.stream(slot.stream):
            slot.start = torch.cuda.Event(enable_timing=True)
            slot.start.record(slot.stream)
            a = torch.as_tensor(req.a, dtype=torch.float64)
            slot.a_dev = a.to("cuda", non_blocking=True) if not a.is_cuda else a
            slot.op.set_material(slot.a_dev)
            slot.op.set_alpha(req.alpha)
            slot.u.zero_()
            st = _lib.lib().pgj_solve_async(slot.op._ctx, self.macros.shape[0], self.macros.ctypes.data, self.rtol,
                                            slot.u.data_ptr(), slot.stream.cuda_stream)
            _lib.check(st, "pgj_solve_async")
            if self.macros.shape[0] == 6:
                _lib.check(_lib.lib().pgj_effective_tensor(slot.op._ctx, slot.u.data_ptr(), slot.C.data_ptr(),
                                                           slot.stream.cuda_stream), "pgj_effective_tensor")
                slot.Ch.copy_(slot.C, non_blocking=True)
            slot.event = torch.cuda.Event(enable_timing=True)
            slot.event.record(slot.stream)
        slot.req = req

    def _collect(self, slot: _Slot) -> Result:
        info = (_lib.LoadInfo * self.macros.shape[0])()
        st = _lib.lib().pgj_solve_wait(slot.op._ctx, info, slot.stream.cuda_stream)
        if st not in (_lib.PGJ_OK, _lib.PGJ_ERR_CERTIFICATION):
            _lib.check(st, "pgj_solve_wait")
        slot.event.synchronize()
        res = Result(slot.req.tag, slot.Ch.numpy().copy(), [i.as_dict() for i in info], st,
                     slot.op.last_refinements(), slot.op.last_launches() + 3, slot.start.elapsed_time(slot.event))
        slot.req = None
        return res

    def streams(self):
        return [s.stream for slots in self.pool.values() for s in slots]

    def warm(self, n: int) -> None:
        """Create the contexts (and tune their tiles) for grid size n ahead of time."""
        self._slots_for(n)

    def run(self, requests: list[Request]) -> list[Result]:
        """Solve all requests; up to `slots` designs of each grid size are in flight at once."""
        pending = list(requests)
        results = []
        busy: list[_Slot] = []
        while pending or busy:
            # fill free slots in request order
            still = []
            for req in pending:
                n = int(np.asarray(req.a).shape[0]) if not hasattr(req.a, "shape") else int(req.a.shape[0])
                free = [s for s in self._slots_for(n) if s.req is None]
                if free:
                    self._launch(free[0], req)
                    busy.append(free[0])
                else:
                    still.append(req)
            pending = still
            # collect the oldest in-flight design (its stream finishes first in FIFO order)
            if busy:
                slot = busy.pop(0)
                results.append(self._collect(slot))
        return results
