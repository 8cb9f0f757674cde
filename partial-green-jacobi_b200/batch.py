"""Concurrent certified homogenizations of many independent designs on one GPU.

Every kernel of one homogenization is latency-bound at n <= 64 (a few waves of small blocks), so one
design cannot fill a B200. ``Batch`` therefore runs ``designs`` designs of the same grid in ONE
batched libpgj context (``pgj_ctx_create_batch``): every kernel launch of the PCG iteration carries
all designs' loads, and the whole certified solve of the group is one graph launch (restarts, PCG
loop and certification decided on the device, per design). ``slots`` such contexts per grid size run
on their own CUDA streams, and designs of different n run side by side. Finished groups are collected
as soon as their stream's event completes, whichever slot that is (no waiting on the oldest group).
A design's result and iteration counts do not depend on its batch-mates: the reductions are per load
in a fixed order and the tile shapes are shared with the one-design context of the same grid.

This is the batched form of the reference's per-design host loop
(``exp/asg_density_selector_20261105/run.py:105-119``), whose only batching is the loads of one design
(``load_mode='parallel'``, ``exp/asg_gpu_resident_20261103/resident.py:72-73``).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .resident import PAPER_MEDIUM


def _torch():
    import torch

    return torch


def _ptr(t) -> int:
    return int(t.data_ptr())


class BatchedOperator:
    """One batched libpgj context: ``designs`` designs of grid n, ``loads`` right-hand sides each."""

    def __init__(self, n: int, designs: int, loads: int, lam: float, mu: float, precision: str = "mixed"):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("partial-green-jacobi_b200 requires a CUDA device (no CPU fallback)")
        L = _lib.lib()
        self.n, self.designs, self.loads = int(n), int(designs), int(loads)
        self.lam, self.mu, self.precision = float(lam), float(mu), precision
        prec = _lib.PGJ_FP32 if precision == "mixed" else _lib.PGJ_FP64
        nbytes = C.c_size_t()
        _lib.check(L.pgj_workspace_bytes_batch(self.n, self.designs, self.loads, prec, C.byref(nbytes)),
                   "pgj_workspace_bytes_batch")
        self.workspace_bytes = nbytes.value
        self._ws = torch.empty(nbytes.value + 256, dtype=torch.uint8, device="cuda")
        base = _ptr(self._ws)
        off = (-base) % 256
        ctx = C.c_void_p()
        _lib.check(L.pgj_ctx_create_batch(self.n, self.designs, self.loads, prec, self.lam, self.mu, base + off,
                                          nbytes.value, torch.cuda.current_stream().cuda_stream, C.byref(ctx)),
                   "pgj_ctx_create_batch")
        self._ctx = ctx
        self._keep = [None] * self.designs

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            try:
                _lib.lib().pgj_ctx_destroy(ctx)
            except Exception:
                pass
            self._ctx = None

    def set_material(self, design: int, a, stream) -> None:
        torch = _torch()
        a = torch.as_tensor(a, dtype=torch.float64)
        if not a.is_cuda:
            a = a.to("cuda", non_blocking=True)
        a = a.contiguous()
        if a.numel() != self.n ** 3:
            raise ValueError("density multiplier must have n^3 entries")
        _lib.check(_lib.lib().pgj_set_material_at(self._ctx, int(design), _ptr(a), stream.cuda_stream),
                   "pgj_set_material_at")
        self._keep[design] = a  # the copy is asynchronous: keep the source alive until it ran

    def set_alpha(self, design: int, alpha: float, stream) -> None:
        _lib.check(_lib.lib().pgj_set_alpha_at(self._ctx, int(design), float(alpha), stream.cuda_stream),
                   "pgj_set_alpha_at")

    def solve_async(self, designs: int, macros: np.ndarray, rtol: float, u, stream) -> None:
        """Enqueue the certified solve of the first ``designs`` designs (u: (designs*loads, 3N))."""
        m = np.ascontiguousarray(np.tile(np.atleast_2d(macros), (designs, 1)), dtype=np.float64)
        self._macros = m  # staged synchronously by the library; kept for symmetry with the infos
        _lib.check(_lib.lib().pgj_solve_async(self._ctx, m.shape[0], m.ctypes.data, float(rtol), _ptr(u),
                                              stream.cuda_stream), "pgj_solve_async")

    def wait(self, designs: int, stream):
        info = (_lib.LoadInfo * (designs * self.loads))()
        st = _lib.lib().pgj_solve_wait(self._ctx, info, stream.cuda_stream)
        if st not in (_lib.PGJ_OK, _lib.PGJ_ERR_CERTIFICATION):
            _lib.check(st, "pgj_solve_wait")
        return [i.as_dict() for i in info], st

    def effective_tensor(self, design: int, u, C6, stream) -> None:
        _lib.check(_lib.lib().pgj_effective_tensor_at(self._ctx, int(design), _ptr(u), _ptr(C6), stream.cuda_stream),
                   "pgj_effective_tensor_at")

    def last_refinements(self) -> int:
        return int(_lib.lib().pgj_last_refinements(self._ctx))

    def last_launches(self) -> int:
        return int(_lib.lib().pgj_last_launches(self._ctx))

    def profile_iteration(self, macros, reps: int = 20):
        """Per-kernel mean durations (ms) and algorithmic bytes of one PCG iteration over all the
        context's designs (CUDA events on the current stream); the designs' fields must be set."""
        m = np.ascontiguousarray(np.tile(np.atleast_2d(macros), (self.designs, 1)), dtype=np.float64)
        ms = (C.c_double * 8)()
        nbytes = (C.c_double * 8)()
        stream = _torch().cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().pgj_profile_iteration(self._ctx, m.shape[0], m.ctypes.data, int(reps), ms, nbytes,
                                                    stream), "pgj_profile_iteration")
        if _lib.lib().pgj_fused_iteration(self._ctx):
            names = ["operator", "update_fft_xy", "fft_z_symbol", "ifft_xy_update_p"]
        else:
            names = ["operator", "update_ur", "fft_x", "fft_y", "fft_z_symbol", "ifft_y", "ifft_x", "update_p"]
        return {k: dict(ms=ms[i], bytes=nbytes[i]) for i, k in enumerate(names)}

    def tile_shapes(self) -> dict:
        out = (C.c_int * 6)()
        _lib.check(_lib.lib().pgj_tile_shapes(self._ctx, out), "pgj_tile_shapes")
        return dict(stencil_rows=out[0], stencil_planes=out[1], fft_rows=out[2], fft_y_columns=out[3],
                    fft_z_columns=out[4], fused=bool(out[5]))


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
    latency_ms: float  # device time from the group's first copy to its C_H on the slot's stream


@dataclass
class _Slot:
    op: BatchedOperator
    stream: object
    u: object
    C: object
    Ch: object
    event: object = None
    start: object = None
    reqs: list | None = None


def _grid(req: Request) -> int:
    a = req.a
    return int(a.shape[0]) if hasattr(a, "shape") else int(np.asarray(a).shape[0])


class Batch:
    """``slots`` batched contexts of ``designs`` designs per grid size, each on its own stream."""

    def __init__(self, slots: int = 2, designs: int = 4, precision: str = "mixed", medium=PAPER_MEDIUM,
                 rtol: float = 1e-8, macros=None):
        self.slots = int(slots)
        self.designs = int(designs)
        self.precision = precision
        self.lam, self.mu = medium
        self.rtol = float(rtol)
        self.macros = np.ascontiguousarray(np.eye(6) if macros is None else np.atleast_2d(macros), dtype=np.float64)
        self.pool: dict[int, list[_Slot]] = {}

    @property
    def loads(self) -> int:
        return self.macros.shape[0]

    def _slots_for(self, n: int) -> list[_Slot]:
        torch = _torch()
        if n not in self.pool:
            slots = []
            for _ in range(self.slots):
                stream = torch.cuda.Stream()
                with torch.cuda.stream(stream):
                    op = BatchedOperator(n, self.designs, self.loads, self.lam, self.mu, self.precision)
                    u = torch.zeros((self.designs * self.loads, 3 * n ** 3), dtype=torch.float64, device="cuda")
                    Cd = torch.empty((self.designs, 6, 6), dtype=torch.float64, device="cuda")
                    Ch = torch.empty((self.designs, 6, 6), dtype=torch.float64).pin_memory()
                slots.append(_Slot(op, stream, u, Cd, Ch))
            torch.cuda.synchronize()
            self.pool[n] = slots
        return self.pool[n]

    def _launch(self, slot: _Slot, reqs: list[Request]) -> None:
        torch = _torch()
        k = len(reqs)
        s = slot.stream
        with torch.cuda.stream(s):
            slot.start = torch.cuda.Event(enable_timing=True)
            slot.start.record(s)
            for d, req in enumerate(reqs):
                slot.op.set_material(d, req.a, s)
                slot.op.set_alpha(d, req.alpha, s)
            u = slot.u[: k * self.loads]
            u.zero_()
            slot.op.solve_async(k, self.macros, self.rtol, u, s)
            if self.loads == 6:
                for d in range(k):
                    slot.op.effective_tensor(d, slot.u[d * 6:(d + 1) * 6], slot.C[d], s)
                slot.Ch[:k].copy_(slot.C[:k], non_blocking=True)
            slot.event = torch.cuda.Event(enable_timing=True)
            slot.event.record(s)
        slot.reqs = reqs

    def _collect(self, slot: _Slot) -> list[Result]:
        k = len(slot.reqs)
        infos, _ = slot.op.wait(k, slot.stream)
        slot.event.synchronize()
        lat = slot.start.elapsed_time(slot.event)
        refinements = slot.op.last_refinements()
        launches = slot.op.last_launches() + 2 * k + k  # + scale builds (2 per design) + C_H
        out = []
        for d, req in enumerate(slot.reqs):
            inf = infos[d * self.loads:(d + 1) * self.loads]
            ok = all(i["converged"] for i in inf)
            out.append(Result(req.tag, slot.Ch[d].numpy().copy(), inf,
                              _lib.PGJ_OK if ok else _lib.PGJ_ERR_CERTIFICATION, refinements, launches // k, lat))
        slot.reqs = None
        for j in range(len(slot.op._keep)):
            slot.op._keep[j] = None
        return out

    def streams(self):
        return [s.stream for slots in self.pool.values() for s in slots]

    def warm(self, n: int) -> None:
        """Create the contexts (and tune their tiles) for grid size n ahead of time."""
        self._slots_for(n)

    def run(self, requests: list[Request]) -> list[Result]:
        """Solve all requests; up to ``slots`` groups of ``designs`` designs per grid size are in
        flight at once. Results come back in completion order."""
        pending: dict[int, list[Request]] = {}
        for req in requests:
            pending.setdefault(_grid(req), []).append(req)
        results: list[Result] = []
        busy: list[_Slot] = []
        while any(pending.values()) or busy:
            for n, queue in pending.items():
                for slot in self._slots_for(n):
                    if not queue:
                        break
                    if slot.reqs is None:
                        group, pending[n] = queue[: self.designs], queue[self.designs:]
                        queue = pending[n]
                        self._launch(slot, group)
                        busy.append(slot)
            # collect every finished group; when none is, poll again shortly
            done = [s for s in busy if s.event.query()]
            if not done and busy:
                time.sleep(2e-4)
                continue
            for slot in done:
                busy.remove(slot)
                results.extend(self._collect(slot))
        return results
