"""Drop-in host classes for the reference's GPU-resident homogenization path.

These keep the call surface of the reference drivers (``examples/shear_design.py``,
``examples/replay_state.py``, ``exp/asg_density_selector_20261105/run.py``):

* ``Operator``          ~ ``HybridFIOperator`` + attached FI Green (``op.apply``, ``op.compute_rhs``,
                           ``op.apply_precond``, ``op.project_zero_mean``, ``op._material_field``)
* ``Resident``          ~ ``exp/asg_gpu_resident_20261103/resident.py:61-213`` (Study I, 3 shear loads)
* ``PaperResident``     ~ ``exp/asg_sctop_reproduction_20261105/reproduction.py:121-176`` (6 Voigt loads)
* ``SelectorResident``  ~ ``exp/asg_density_selector_20261105/run.py:46-77`` (choose + build_scale)

Every numerical step runs in libpgj (hand-written sm_100a kernels) through its C ABI; PyTorch only
provides device memory and the current stream, except the alpha selectors of ``SelectorResident``
(one scalar per design from a few reductions over the density, ``alpha_selectors.py``). Device
buffers are owned here (torch tensors) and lent to the library by pointer.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib, alpha_selectors as selectors
from .outer import PaperOuter, ResidentOuter

STUDY1_MEDIUM = (4.0 / 3.0, 1.0)
PAPER_MEDIUM = (15.0 / 26.0, 5.0 / 13.0)
# calibrated eta-lookup exponents per weak-material ratio (reference MODELS_FROZEN.json models.eta)
ETA_ANCHORS = {1e-4: 9 / 16, 1e-6: 11 / 16, 1e-9: 13 / 16}


def _torch():
    import torch

    return torch


def _stream_ptr():
    return _torch().cuda.current_stream().cuda_stream


def _ptr(t) -> int:
    return int(t.data_ptr())


class Backend:
    """Study I medium (lambda=4/3, mu=1) and the three unit engineering shears (backend.py:58-60,102)."""

    def __init__(self):
        lam, mu = STUDY1_MEDIUM
        self.lam, self.mu = lam, mu
        self.C0 = _c0(lam, mu)
        self.loads = np.eye(6)[3:]


class PaperBackend(Backend):
    """Paper medium E=1, nu=0.3 (lambda=15/26, mu=5/13) and the six unit Voigt strains (reproduction.py:56-66)."""

    def __init__(self):
        lam, mu = PAPER_MEDIUM
        self.lam, self.mu = lam, mu
        self.C0 = _c0(lam, mu)
        self.loads = np.eye(6)


def _c0(lam, mu):
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[np.arange(3), np.arange(3)] += 2 * mu
    c[np.arange(3, 6), np.arange(3, 6)] = mu
    return c


def _medium(backend):
    c0 = np.asarray(backend.C0, dtype=np.float64)
    lam, mu = float(c0[0, 1]), float(c0[3, 3])
    expected = _c0(lam, mu)
    if not np.allclose(expected, c0, rtol=1e-14, atol=0):
        raise ValueError("isotropic C0 required")
    return lam, mu


class Operator:
    """Periodic HEX8 operator + FI Green preconditioner on one grid, over a libpgj context.

    ``loads`` is the number of simultaneous right-hand sides the context holds. ``precision`` is
    ``"fp64"`` (plain) or ``"mixed"`` (FP32 inner operator/Green/PCG inside FP64 refinement).
    """

    def __init__(self, n: int, loads: int, lam: float, mu: float, precision: str = "fp64"):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("partial-green-jacobi_b200 requires a CUDA device (no CPU fallback)")
        L = _lib.lib()
        self.n, self.loads, self.lam, self.mu = int(n), int(loads), float(lam), float(mu)
        self.precision = precision
        prec = _lib.PGJ_FP32 if precision == "mixed" else _lib.PGJ_FP64
        nbytes = C.c_size_t()
        _lib.check(L.pgj_workspace_bytes(self.n, self.loads, prec, C.byref(nbytes)), "pgj_workspace_bytes")
        self._ws = torch.empty(nbytes.value + 256, dtype=torch.uint8, device="cuda")
        base = _ptr(self._ws)
        self._off = (-base) % 256
        ctx = C.c_void_p()
        _lib.check(L.pgj_ctx_create(self.n, self.loads, prec, self.lam, self.mu, base + self._off, nbytes.value,
                                    _stream_ptr(), C.byref(ctx)), "pgj_ctx_create")
        self._ctx = ctx
        N = self.n ** 3
        self.solutions = self._view(L.pgj_ctx_solutions(ctx), (self.loads, 3 * N))
        self.scale = self._view(L.pgj_ctx_scale(ctx), (1, 3 * N))
        self._material_field = self._view(L.pgj_ctx_material(ctx), (self.n, self.n, self.n))
        self.mesh_shape = (self.n,) * 3

    def _view(self, ptr, shape):
        torch = _torch()
        start = int(ptr) - _ptr(self._ws)
        count = int(np.prod(shape))
        return self._ws[start:start + 8 * count].view(torch.float64).view(*shape)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            try:
                _lib.lib().pgj_ctx_destroy(ctx)
            except Exception:
                pass
            self._ctx = None

    # --- state -------------------------------------------------------------------------------
    def set_material(self, a) -> None:
        torch = _torch()
        a = torch.as_tensor(a, dtype=torch.float64, device="cuda").contiguous()
        if a.numel() != self.n ** 3:
            raise ValueError("density multiplier must have n^3 entries")
        _lib.check(_lib.lib().pgj_set_material(self._ctx, _ptr(a), _stream_ptr()), "pgj_set_material")
        self._keep = a

    def set_alpha(self, alpha: float) -> None:
        _lib.check(_lib.lib().pgj_set_alpha(self._ctx, float(alpha), _stream_ptr()), "pgj_set_alpha")

    # --- operator surface (HybridFIOperator) ----------------------------------------------------
    def _check_vec(self, u, dtype=None):
        torch = _torch()
        dtype = dtype or torch.float64
        if u.dtype != dtype or not u.is_cuda or not u.is_contiguous() or u.dim() != 2 or u.shape[1] != 3 * self.n ** 3:
            raise ValueError(f"expected contiguous CUDA {dtype} (L, 3N) vectors")
        if u.shape[0] > self.loads:
            raise ValueError("more vectors than the context holds")

    def apply(self, u, active=None):
        torch = _torch()
        if u.dtype == torch.float32:
            self._check_vec(u, torch.float32)
            fn = _lib.lib().pgj_apply_f32
        else:
            self._check_vec(u)
            fn = _lib.lib().pgj_apply
        q = torch.empty_like(u)
        act = 0
        if active is not None:
            active = torch.as_tensor(active, device="cuda").to(torch.int32).contiguous()
            act = _ptr(active)
        _lib.check(fn(self._ctx, u.shape[0], _ptr(u), act, _ptr(q), _stream_ptr()), "pgj_apply")
        return q

    def compute_rhs(self, macro):
        torch = _torch()
        m = np.ascontiguousarray(np.atleast_2d(np.asarray(macro, dtype=np.float64)))
        if m.shape[1] != 6:
            raise ValueError("six engineering macro strain components required")
        f = torch.empty((m.shape[0], 3 * self.n ** 3), dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().pgj_rhs(self._ctx, m.shape[0], m.ctypes.data, _ptr(f), _stream_ptr()), "pgj_rhs")
        return f

    def apply_precond(self, r):
        torch = _torch()
        self._check_vec(r)
        z = torch.empty_like(r)
        _lib.check(_lib.lib().pgj_precondition(self._ctx, r.shape[0], _ptr(r), _ptr(z), _stream_ptr()),
                   "pgj_precondition")
        return z

    def project_zero_mean(self, value):
        q = value.view(value.shape[0], -1, 3)
        return (q - q.mean(dim=1, keepdim=True)).reshape(value.shape[0], -1)

    # --- solve / responses ----------------------------------------------------------------------
    def solve(self, macros, rtol: float, u):
        """Certified solve of ``len(macros)`` loads in place on ``u`` (L, 3N). Returns (infos, status)."""
        m = np.ascontiguousarray(np.atleast_2d(np.asarray(macros, dtype=np.float64)))
        self._check_vec(u)
        if u.shape[0] != m.shape[0]:
            raise ValueError("one macro strain per load")
        info = (_lib.LoadInfo * m.shape[0])()
        st = _lib.lib().pgj_solve(self._ctx, m.shape[0], m.ctypes.data, float(rtol), _ptr(u), info, _stream_ptr())
        if st not in (_lib.PGJ_OK, _lib.PGJ_ERR_CERTIFICATION):
            _lib.check(st, "pgj_solve")
        return [i.as_dict() for i in info], st

    def set_inner_rtol(self, rtol: float) -> None:
        _lib.check(_lib.lib().pgj_set_inner_rtol(self._ctx, float(rtol)), "pgj_set_inner_rtol")

    def set_mixed_mode(self, mode: str = "reliable", delta: float = 0.1) -> None:
        """``"reliable"``: one FP32 recurrence with FP64 true-residual replacements; ``"sweeps"``:
        restarted refinement sweeps."""
        m = {"reliable": 0, "sweeps": 1}[mode]
        _lib.check(_lib.lib().pgj_set_mixed_mode(self._ctx, m, float(delta)), "pgj_set_mixed_mode")

    def set_iteration_cap(self, cap: int) -> None:
        """Per-load PCG iteration cap (default 4000, the reference's)."""
        _lib.check(_lib.lib().pgj_set_iteration_cap(self._ctx, int(cap)), "pgj_set_iteration_cap")

    def set_flexible_beta(self, on: bool) -> None:
        """Mixed contexts: Polak-Ribiere direction updates of the FP32 recurrences."""
        _lib.check(_lib.lib().pgj_set_flexible_beta(self._ctx, 1 if on else 0), "pgj_set_flexible_beta")

    def set_mixed_operator(self, fp64: bool) -> None:
        """Mixed contexts: run the recurrence operator in FP64 arithmetic on the FP32 vectors
        (for weak-material ratios near 1e-9, where FP32 node sums of stiff and weak elements cancel)."""
        _lib.check(_lib.lib().pgj_set_mixed_operator(self._ctx, 1 if fp64 else 0), "pgj_set_mixed_operator")

    def last_refinements(self) -> int:
        return int(_lib.lib().pgj_last_refinements(self._ctx))

    def last_launches(self) -> int:
        return int(_lib.lib().pgj_last_launches(self._ctx))

    def profile_iteration(self, macros, reps: int = 20):
        """Per-kernel mean durations (ms) and algorithmic bytes of one PCG iteration (CUDA events)."""
        m = np.ascontiguousarray(np.atleast_2d(np.asarray(macros, dtype=np.float64)))
        ms = (C.c_double * 8)()
        nbytes = (C.c_double * 8)()
        _lib.check(_lib.lib().pgj_profile_iteration(self._ctx, m.shape[0], m.ctypes.data, int(reps), ms, nbytes,
                                                    _stream_ptr()), "pgj_profile_iteration")
        if self.fused_iteration:
            names = ["operator", "update_fft_xy", "fft_z_symbol", "ifft_xy_update_p"]
        else:
            names = ["operator", "update_ur", "fft_x", "fft_y", "fft_z_symbol", "ifft_y", "ifft_x", "update_p"]
        return {k: dict(ms=ms[i], bytes=nbytes[i]) for i, k in enumerate(names)}

    def tile_shapes(self) -> dict:
        """Tile shapes picked by the operator and Green-pass autotuners for this context."""
        out = (C.c_int * 6)()
        _lib.check(_lib.lib().pgj_tile_shapes(self._ctx, out), "pgj_tile_shapes")
        return dict(stencil_rows=out[0], stencil_planes=out[1], fft_rows=out[2], fft_y_columns=out[3],
                    fft_z_columns=out[4], fused=bool(out[5]))

    @property
    def fused_iteration(self) -> bool:
        """True when one PCG iteration runs as four kernels (slab-fused updates and transforms)."""
        return bool(_lib.lib().pgj_fused_iteration(self._ctx))

    def set_fused_iteration(self, on: bool) -> None:
        _lib.check(_lib.lib().pgj_set_fused_iteration(self._ctx, 1 if on else 0), "pgj_set_fused_iteration")

    def energies(self, u, macros):
        torch = _torch()
        m = np.ascontiguousarray(np.atleast_2d(np.asarray(macros, dtype=np.float64)))
        self._check_vec(u)
        e = torch.empty((u.shape[0], self.n ** 3), dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().pgj_energies(self._ctx, u.shape[0], _ptr(u), m.ctypes.data, _ptr(e), _stream_ptr()),
                   "pgj_energies")
        return e

    def effective_tensor(self, u):
        torch = _torch()
        if u.shape != (6, 3 * self.n ** 3) or u.dtype != torch.float64 or not u.is_contiguous():
            raise ValueError("six contiguous FP64 Voigt solutions required")
        C6 = torch.empty((6, 6), dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().pgj_effective_tensor(self._ctx, _ptr(u), _ptr(C6), _stream_ptr()), "pgj_effective_tensor")
        return C6


class Resident:
    """Study I solver: three unit shear loads, FP64 PCG with certification (resident.py:61-213)."""

    n_loads = 3

    def __init__(self, backend=None, n=32, chunk=4, load_mode="serial", precision="fp64"):
        torch = _torch()
        backend = backend or Backend()
        if chunk < 1:
            raise ValueError("positive graph chunk required")
        if load_mode not in ("serial", "parallel"):
            raise ValueError("load_mode must be serial or parallel")
        self.b = backend
        self.n = int(n)
        self.chunk = chunk
        self.load_mode = load_mode
        self.batch = 1 if load_mode == "serial" else self.n_loads
        self.lam, self.mu = _medium(backend)
        self.macros = np.asarray(backend.loads, dtype=np.float64)[: self.n_loads]
        self.op = Operator(self.n, self.n_loads, self.lam, self.mu, precision)
        self.solutions = self.op.solutions
        self.scale = self.op.scale
        self.alpha = torch.zeros((), device="cuda", dtype=torch.float64)
        self.outer = self._make_outer()

    def _make_outer(self):
        return ResidentOuter(self.n)

    def capture(self):
        self.outer.capture()
        self.solutions.zero_()

    def material(self, a):
        self.op.set_material(a)

    def select(self, method):
        if method == "green":
            alpha = 0.0
        elif method == "gj":
            alpha = 1.0
        elif method == "compact8":
            # compact law on the density field (exp/asg_gpu_resident_20261103/resident.py:163-168)
            alpha = float(selectors.compact8_alpha(self.op._material_field))
        elif method == "asg":
            # frozen ASG MLP on the density field's statistics (resident.py:160-162)
            alpha = float(selectors.asg_alpha(self.op._material_field))
        else:
            try:
                alpha = float(method)
            except (TypeError, ValueError):
                raise ValueError(f"unsupported preconditioner selection {method!r}") from None
        self.alpha.fill_(alpha)
        self.op.set_alpha(alpha)

    def solve(self, rtol=1e-8):
        infos = []
        checks = 0
        loads = range(self.n_loads)
        groups = [list(loads)] if self.batch > 1 else [[l] for l in loads]
        for g in groups:
            u = self.solutions[g[0]:g[-1] + 1]
            info, st = self.op.solve(self.macros[g[0]:g[-1] + 1], rtol, u)
            infos.extend(info)
            checks += 1 + max(i["restarts"] for i in info)
            if st == _lib.PGJ_ERR_CERTIFICATION:
                raise RuntimeError(("true residual certification failed", info))
        return infos, checks

    def energy(self):
        e = self.op.energies(self.solutions, self.macros)
        a = self.op._material_field.reshape(1, -1)
        return (e * a).mean(1), e.mean(0).reshape(self.n, self.n, self.n)


class PaperResident(Resident):
    """Six-load (Voigt) solver with the paper medium and the SCTOP outer loop (reproduction.py:121-176)."""

    n_loads = 6

    def __init__(self, backend=None, n=32, objective="shear", volume=0.2, rmin=3.0, beta=4.0, eta=0.5, emin=1e-9,
                 load_mode="parallel", chunk=4, precision="fp64"):
        self._outer_args = (volume, rmin, beta, eta, emin)
        self.objective_kind = objective
        super().__init__(backend or PaperBackend(), n, chunk, load_mode, precision)

    def _make_outer(self):
        volume, rmin, beta, eta, emin = self._outer_args
        return PaperOuter(self.n, volume, rmin, beta, eta, emin)

    def energy(self, iteration=0):
        torch = _torch()
        e = self.op.energies(self.solutions, self.macros)
        a = self.op._material_field.reshape(1, -1)
        diagonal = (e * a).mean(1)
        if self.objective_kind == "shear":
            local = -e[3:].sum(0)
        else:
            hydro_u = self.solutions[:3].sum(0, keepdim=True).contiguous()
            hydro = self.op.energies(hydro_u, [[1.0, 1.0, 1.0, 0.0, 0.0, 0.0]])[0]
            if self.objective_kind == "bulk":
                local = -hydro
            elif self.objective_kind == "auxetic":
                local = hydro - (1 + 0.8 ** iteration) * e[:3].sum(0)
            else:
                raise ValueError(self.objective_kind)
        objective = (local * a.reshape(-1)).mean()
        return objective, local.reshape(self.n, self.n, self.n), diagonal

    def effective_tensor(self):
        return self.op.effective_tensor(self.solutions)


class SelectorResident(PaperResident):
    """``choose`` (alpha) + ``build_scale`` (D^-alpha/2) as separate steps (run.py:46-77).

    Methods: green, gj, eta (lookup by Emin), contrast, gray, compact8, compact8q, or a number.
    The selectors are small reductions over the density on the device (``alpha_selectors.py``).
    """

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        emin = self.outer.emin
        self.eta_value = ETA_ANCHORS[min(ETA_ANCHORS, key=lambda k: abs(math.log10(k) - math.log10(emin)))]
        self.contrast_anchors = selectors.CONTRAST_ANCHORS

    def choose(self, method):
        a = self.op._material_field
        if method == "green":
            self.alpha.zero_()
        elif method == "gj":
            self.alpha.fill_(1.0)
        elif method == "eta":
            self.alpha.fill_(self.eta_value)
        elif method == "contrast":
            self.alpha.copy_(selectors.contrast_alpha(a, self.contrast_anchors))
        elif method == "gray":
            self.alpha.copy_(selectors.gray_alpha(a, self.outer.ph))
        elif method in ("compact8", "compact8q"):
            self.alpha.copy_(selectors.compact8_alpha(a, quantize=method == "compact8q"))
        else:
            try:
                self.alpha.fill_(float(method))
            except (TypeError, ValueError):
                raise ValueError(f"unsupported preconditioner selection {method!r}") from None

    def build_scale(self, method):
        alpha = 0.0 if method == "green" else float(self.alpha)
        self.op.set_alpha(alpha)

    def select(self, method):
        self.choose(method)
        self.build_scale(method)
