"""CPU oracle for the periodic HEX8 homogenization hot path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product path (``partial-green-jacobi_b200``) runs on hand-written CUDA kernels and
fails loudly when its shared library is missing.

It restates, in vectorised NumPy/SciPy, the arithmetic of the reference
(yufangjie1643/partial-green-jacobi). Each function cites the reference file:line it
follows:

* element stiffness, exact 2x2x2 Gauss Q1/HEX8 ... ``exp/asg_candidates_20261103/candidates.py:31-54``
  (the modal form ``solver/src/materials/fi_modal.cuh:2-255`` computes the same product)
* operator K(a) u = sum_e a_e Ke u_e ........... ``exp/asg_gpu_resident_20261103/scalar_fi.cu:14-36``
* right-hand side f = -V sum B_c^T C eps ........ ``solver/src/materials/hybrid_kernels.cu:50-68``
* FI Green symbol, dense 6-coefficient form ..... ``solver/src/reference_medium/formula_kernels.cu:104-126``,
  ``solver/src/reference_medium/formula_adapter.py:48-53``, ``solver/src/spectral/precision_kernels.cu:57-89``
* Green apply (rfftn -> symbol -> irfftn) ........ ``exp/asg_gpu_resident_20261103/resident.py:109-117``,
  ``exp/asg_gpu_resident_20261103/scalar_fi.cu:38-44``
* stiffness diagonal and D^-alpha/2 scaling ...... ``solver/experiments/smooth_contrast/study.py:56-66``,
  ``exp/asg_gpu_resident_20261103/resident.py:156-174``
* masked multi-load PCG, certification, restarts . ``exp/asg_gpu_resident_20261103/resident.py:28-58,119-136,186-209``
* energies, affine fields, C_H ................... ``exp/asg_scenarios_20261105/energy.cu:7-24``,
  ``exp/asg_topopt_20261103/backend.py:153-162``, ``exp/asg_sctop_reproduction_20261105/reproduction.py:153-176``
* Study I generator / filter / OC ............... ``exp/asg_topopt_20261103/study.py:61-100``,
  ``exp/asg_gpu_resident_20261103/outer.py:12-59``, ``exp/asg_gpu_resident_20261103/outer.cu:7-37``
* Study II cone filter / projection / OC ......... ``exp/asg_sctop_reproduction_20261105/reproduction.py:38-118``,
  ``exp/asg_sctop_reproduction_20261105/outer.cu:8-39``
* alpha selectors (contrast, gray, compact8) ...... ``exp/asg_density_selector_20261105/run.py:27-43,53-67``,
  ``solver/experiments/global_alpha_compact_law/law.py:10-19``

Layouts follow the reference: a DOF vector is (L, 3N) float64, node-major with the xyz
components interleaved, nodes in grid order (z, y, x); a scalar field is (n, n, n) in
(z, y, x) order. Element e=(x,y,z) owns the nodes (x+bx, y+by, z+bz) with the local index
b = bx + 2 by + 4 bz.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# Study I application medium (lambda=4/3, mu=1) and Study II / paper medium (E=1, nu=0.3).
STUDY1 = (4.0 / 3.0, 1.0)
PAPER = (15.0 / 26.0, 5.0 / 13.0)
ITERATION_CAP = 4000


# ----------------------------------------------------------------------------- element
def c0_matrix(lam: float, mu: float) -> np.ndarray:
    """Isotropic 6x6 Voigt stiffness (xx, yy, zz, yz, xz, xy; engineering shear)."""
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[np.arange(3), np.arange(3)] += 2 * mu
    c[np.arange(3, 6), np.arange(3, 6)] = mu
    return c


def packed21(lam: float, mu: float) -> np.ndarray:
    """Upper-triangular row-major 21-vector of C0 (``backend.py:101``)."""
    c = c0_matrix(lam, mu)
    return np.array([c[i, j] for i in range(6) for j in range(i, 6)])


def local_offsets() -> np.ndarray:
    """Local node offsets (bx, by, bz) in bit order b = bx + 2by + 4bz (``scalar_fi.cu:25``)."""
    return np.array([[b & 1, (b >> 1) & 1, (b >> 2) & 1] for b in range(8)])


def element_stiffness(n: int, lam: float, mu: float) -> np.ndarray:
    """24x24 Q1 element stiffness for voxel h=1/n, 2x2x2 Gauss (``candidates.py:31-54``)."""
    off = local_offsets()
    pts = np.array([[x, y, z] for z in (-1, 1) for y in (-1, 1) for x in (-1, 1)]) / (2 * np.sqrt(3)) + 0.5
    c = c0_matrix(lam, mu)
    ke = np.zeros((24, 24))
    for p in pts:
        bmat = np.zeros((6, 24))
        for a, v in enumerate(off):
            fac = np.where(v, p, 1 - p)
            g = [(2 * v[d] - 1) * np.prod(np.delete(fac, d)) * n for d in range(3)]
            dx, dy, dz = g
            bmat[0, 3 * a] = dx
            bmat[1, 3 * a + 1] = dy
            bmat[2, 3 * a + 2] = dz
            bmat[3, 3 * a + 1] = dz
            bmat[3, 3 * a + 2] = dy
            bmat[4, 3 * a] = dz
            bmat[4, 3 * a + 2] = dx
            bmat[5, 3 * a] = dy
            bmat[5, 3 * a + 1] = dx
        ke += bmat.T @ c @ bmat
    return ke / n ** 3 / 8


def element_diagonal(n: int, lam: float, mu: float) -> np.ndarray:
    """(8, 3) diagonal of Ke per local node (``smooth_contrast/study.py:56-66``), bit order."""
    return np.diag(element_stiffness(n, lam, mu)).reshape(8, 3).copy()


# ----------------------------------------------------------------------------- grid helpers
def _as_nodes(v: np.ndarray, n: int) -> np.ndarray:
    return v.reshape(v.shape[0], n, n, n, 3)


def _gather(u5: np.ndarray) -> np.ndarray:
    """(L,n,n,n,3) node field -> (L,N,24) element DOFs: U[e, 3b+c] = u[e+b, c]."""
    cols = []
    for bx, by, bz in local_offsets():
        cols.append(np.roll(u5, shift=(-bz, -by, -bx), axis=(1, 2, 3)))
    stacked = np.stack(cols, axis=4)  # (L,n,n,n,8,3)
    return stacked.reshape(u5.shape[0], -1, 24)


def _scatter(fe: np.ndarray, n: int, reverse: bool = False) -> np.ndarray:
    """(L,N,24) element forces -> (L,3N) node forces: q[node] = sum_b F[node-b, b].

    ``reverse`` sums the eight corners in the opposite order (same value, other rounding).
    """
    L = fe.shape[0]
    f6 = fe.reshape(L, n, n, n, 8, 3)
    out = np.zeros((L, n, n, n, 3))
    corners = list(enumerate(local_offsets()))
    for b, (bx, by, bz) in (corners[::-1] if reverse else corners):
        out += np.roll(f6[:, :, :, :, b, :], shift=(bz, by, bx), axis=(1, 2, 3))
    return out.reshape(L, -1)


def apply_operator(a: np.ndarray, u: np.ndarray, lam: float, mu: float,
                   active: np.ndarray | None = None, reverse: bool = False) -> np.ndarray:
    """q = K(a) u for each load; inactive loads return zeros (``scalar_fi.cu:14-36``)."""
    n = a.shape[0]
    u = np.atleast_2d(u)
    ke = element_stiffness(n, lam, mu)
    ue = _gather(_as_nodes(u, n))
    fe = (ue @ ke) * a.reshape(1, -1, 1)
    q = _scatter(fe, n, reverse)
    if active is not None:
        q[~np.asarray(active, bool)] = 0.0
    return q


_REF_MODAL = None


def apply_operator_ref(a: np.ndarray, u: np.ndarray, lam: float, mu: float,
                       active: np.ndarray | None = None) -> np.ndarray:
    """q = K(a) u with the reference's own element arithmetic: the exact modal element action of
    ``solver/src/materials/fi_modal.cuh:2-255`` on C0, times a_e, summed into the nodes
    (``exp/asg_gpu_resident_20261103/scalar_fi.cu:14-36``). The header is compiled on the host by
    ``oracle/Makefile`` into ``oracle/_ref/libref_fi_modal.so`` (this container only)."""
    global _REF_MODAL
    import ctypes
    from pathlib import Path

    if _REF_MODAL is None:
        _REF_MODAL = ctypes.CDLL(str(Path(__file__).resolve().parent / "_ref" / "libref_fi_modal.so"))
        _REF_MODAL.ref_fi_modal_batch.restype = None
    n = a.shape[0]
    u = np.atleast_2d(u)
    ue = np.ascontiguousarray(_gather(_as_nodes(u, n)))
    fe = np.empty_like(ue)
    c21 = np.ascontiguousarray(packed21(lam, mu))
    h = 1.0 / n
    g = np.array([1 / (4 * h)] * 3 + [h ** 3])
    vp = ctypes.c_void_p
    _REF_MODAL.ref_fi_modal_batch(vp(ue.ctypes.data), vp(c21.ctypes.data), vp(g.ctypes.data), vp(fe.ctypes.data),
                                  ctypes.c_long(ue.shape[0] * ue.shape[1]))
    fe *= a.reshape(1, -1, 1)
    q = _scatter(fe, n)
    if active is not None:
        q[~np.asarray(active, bool)] = 0.0
    return q


def rhs(a: np.ndarray, macro: np.ndarray, lam: float, mu: float) -> np.ndarray:
    """Periodic nodal forces f = -V sum_{8 el} B_c^T (a_e C0) eps (``hybrid_kernels.cu:50-68``)."""
    n = a.shape[0]
    macro = np.atleast_2d(np.asarray(macro, dtype=np.float64))
    c = c0_matrix(lam, mu)
    h = 1.0 / n
    gx = 1.0 / (4 * h)
    vol = h ** 3
    out = np.zeros((macro.shape[0], n, n, n, 3))
    for li, m in enumerate(macro):
        s0 = c @ m  # stress per unit a
        for bx, by, bz in local_offsets():
            # node = e + b, element e = node - b
            ae = np.roll(a, shift=(bz, by, bx), axis=(0, 1, 2))
            dx = gx if bx else -gx
            dy = gx if by else -gx
            dz = gx if bz else -gx
            s = ae[..., None] * s0  # (n,n,n,6)
            out[li, ..., 0] -= vol * (dx * s[..., 0] + dy * s[..., 5] + dz * s[..., 4])
            out[li, ..., 1] -= vol * (dx * s[..., 5] + dy * s[..., 1] + dz * s[..., 3])
            out[li, ..., 2] -= vol * (dx * s[..., 4] + dy * s[..., 3] + dz * s[..., 2])
    return out.reshape(macro.shape[0], -1)


def project(v: np.ndarray) -> np.ndarray:
    """P: remove the per-component mean over nodes (``resident.py:28-31``)."""
    q = v.reshape(v.shape[0], -1, 3)
    return (q - q.mean(1, keepdims=True)).reshape(v.shape)


# ----------------------------------------------------------------------------- Green symbol
def green_symbol(n: int, lam: float, mu: float) -> np.ndarray:
    """Dense (6, n, n, n//2+1) real symbol of the FI HEX8 Green operator, 1/N folded in.

    Steps of ``formula_kernels.cu:104-126`` (diagonal + rank-1 inverse) expanded as in
    ``precision_kernels.cu:57-89`` (dense mode). Coefficient order: xx, yy, zz, xy, xz, yz.
    Half-angle tables theta_i = pi k_i / n (``formula_adapter.py:32-53``).
    """
    h = 1.0 / n
    ns = n // 2 + 1
    tx = np.pi * np.arange(ns) / n
    ty = np.pi * np.arange(n) / n
    tz = np.pi * np.arange(n) / n
    TZ, TY, TX = np.meshgrid(tz, ty, tx, indexing="ij")
    s = [np.sin(TX), np.sin(TY), np.sin(TZ)]
    c = [np.cos(TX), np.cos(TY), np.cos(TZ)]
    m = [c[i] * c[i] + s[i] * s[i] / 3 for i in range(3)]
    t = h * h * h * m[0] * m[1] * m[2]
    v = [2 * s[i] * c[i] / (h * m[i]) for i in range(3)]
    d = [4 * s[i] ** 4 / (3 * h * h * m[i] * m[i]) for i in range(3)]
    trace = t * ((d[0] + v[0] ** 2) + (d[1] + v[1] ** 2) + (d[2] + v[2] ** 2))
    b = (lam + mu) * t
    zero = np.zeros_like(t, dtype=bool)
    zero[0, 0, 0] = True
    inv = []
    den = np.ones_like(t)
    with np.errstate(divide="ignore", invalid="ignore"):
        for i in range(3):
            q = np.where(zero, 0.0, 1.0 / (mu * trace + (lam + mu) * t * d[i]))
            inv.append(q)
            den = den + b * v[i] * v[i] * q
        beta = np.where(zero, 0.0, b / den)
    inv_n = 1.0 / float(n ** 3)
    w = [inv[i] * v[i] for i in range(3)]
    out = np.empty((6, n, n, ns))
    out[0] = (inv[0] - beta * w[0] * w[0]) * inv_n
    out[1] = (inv[1] - beta * w[1] * w[1]) * inv_n
    out[2] = (inv[2] - beta * w[2] * w[2]) * inv_n
    out[3] = -beta * w[0] * w[1] * inv_n
    out[4] = -beta * w[0] * w[2] * inv_n
    out[5] = -beta * w[1] * w[2] * inv_n
    return out


def _fft_workers() -> int:
    return int(os.environ.get("PGJ_ORACLE_THREADS", os.cpu_count() or 1))


def green_unscaled(v: np.ndarray, symbol: np.ndarray) -> np.ndarray:
    """z = irfftn(G_hat . rfftn(v)) for each load (``resident.py:111-116``, ``scalar_fi.cu:38-44``)."""
    import scipy.fft as sfft

    L = v.shape[0]
    n = symbol.shape[1]
    field = v.reshape(L, n, n, n, 3).transpose(0, 4, 1, 2, 3)
    spec = sfft.rfftn(field, axes=(-3, -2, -1), workers=_fft_workers())
    x, y, z = spec[:, 0], spec[:, 1], spec[:, 2]
    c0, c1, c2, c3, c4, c5 = symbol
    out = np.empty_like(spec)
    out[:, 0] = c0 * x + c3 * y + c4 * z
    out[:, 1] = c3 * x + c1 * y + c5 * z
    out[:, 2] = c4 * x + c5 * y + c2 * z
    w = sfft.irfftn(out, s=(n, n, n), axes=(-3, -2, -1), norm="forward", workers=_fft_workers())
    return np.ascontiguousarray(w.transpose(0, 2, 3, 4, 1)).reshape(L, -1)


# ----------------------------------------------------------------------------- scaling
def stiffness_diagonal(a: np.ndarray, lam: float, mu: float) -> np.ndarray:
    """d(node, c) = sum_b a(node - b) diag(Ke)[b, c] (``adaptive_green_scaling/study.py:80-89``)."""
    n = a.shape[0]
    ed = element_diagonal(n, lam, mu)
    d = np.zeros((n, n, n, 3))
    for b, (bx, by, bz) in enumerate(local_offsets()):
        d += np.roll(a, shift=(bz, by, bx), axis=(0, 1, 2))[..., None] * ed[b]
    return d.reshape(1, -1)


def scale_field(a: np.ndarray, alpha: float, lam: float, mu: float) -> np.ndarray:
    """D^-alpha/2 with D normalised by its geometric mean (``resident.py:170-174``)."""
    n = a.shape[0]
    if alpha == 0.0:
        return np.ones((1, 3 * n ** 3))
    q = np.log(stiffness_diagonal(a, lam, mu))
    q = q - q.mean()
    return np.exp((-0.5 * alpha) * q)


def precondition(r: np.ndarray, scale: np.ndarray, symbol: np.ndarray) -> np.ndarray:
    """M_alpha^-1 r = P(s . G(s . P r)) (``resident.py:33-37,104-117``)."""
    v = project(r) * scale
    return project(green_unscaled(v, symbol) * scale)


# ----------------------------------------------------------------------------- PCG
@dataclass
class SolveInfo:
    rhs_norm: float
    absolute_residual: float
    threshold: float
    iterations: int
    relative_residual: float
    converged: bool
    restarts: int

    def as_dict(self) -> dict:
        return dict(self.__dict__)


@dataclass
class Problem:
    """Design + medium + preconditioner data shared by all loads."""
    a: np.ndarray
    lam: float
    mu: float
    alpha: float
    scale: np.ndarray = field(init=False)
    symbol: np.ndarray = field(init=False)

    def __post_init__(self):
        self.a = np.ascontiguousarray(self.a, dtype=np.float64)
        self.scale = scale_field(self.a, self.alpha, self.lam, self.mu)
        self.symbol = green_symbol(self.a.shape[0], self.lam, self.mu)

    @property
    def n(self) -> int:
        return self.a.shape[0]

    reverse: bool = False
    ref_arith: bool = False

    def K(self, u, active=None):
        if self.ref_arith:
            return apply_operator_ref(self.a, u, self.lam, self.mu, active)
        return apply_operator(self.a, u, self.lam, self.mu, active, self.reverse)

    def B(self, r):
        return precondition(r, self.scale, self.symbol)


def _dot_a(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    return (x * y).sum(1)


def _dot_b(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """The same per-load dot product summed per component first, z before x (other rounding)."""
    part = (x * y).reshape(x.shape[0], -1, 3).sum(1)
    return part[:, 2] + part[:, 1] + part[:, 0]


def solve_batch(prob: Problem, f: np.ndarray, u0: np.ndarray | None = None, rtol: float = 1e-8,
                max_restarts: int = 2, iteration_cap: int = ITERATION_CAP, max_iterations: int | None = None,
                order: str = "a"):
    """Masked multi-load PCG with true-residual certification (``resident.py:119-136,186-209``).

    ``order`` "b" runs the same recurrence with the recurrence dot products and the operator's
    corner sums in another order: equal in exact arithmetic, rounded differently. An iteration
    count that agrees between the two orders is stable against rounding-level perturbations.
    ``order`` "r" evaluates the operator with the reference's own modal element arithmetic
    (``apply_operator_ref``) instead of the dense 24 x 24 element product.

    ``max_iterations`` bounds the total PCG iterations run (timing samples only); a bounded run
    returns whatever state it reached.
    Returns (u, infos, raised) where ``raised`` is True when the reference would raise
    ``RuntimeError('true residual certification failed', info)``.
    """
    L = f.shape[0]
    n = prob.n
    dot = {"a": _dot_a, "b": _dot_b, "r": _dot_a}[order]
    prob.reverse = order == "b"
    prob.ref_arith = order == "r"
    u = np.zeros_like(f) if u0 is None else np.array(u0, dtype=np.float64)
    norm = np.sqrt((f * f).sum(1))
    target2 = np.maximum(norm * rtol, np.full_like(norm, 1e-13 / math.sqrt(n))) ** 2
    iterations = np.zeros(L, dtype=np.int64)
    bad = np.zeros(L, dtype=bool)

    def certify(u):
        u = project(u)
        r = f - prob.K(u)
        return u, r, np.sqrt((r * r).sum(1))

    u, r, absolute = certify(u)
    restarts = 0
    total = 0
    while True:
        active = (dot(r, r) > target2) & (iterations < iteration_cap) & ~bad
        z = prob.B(r)
        p = np.where(active[:, None], z, 0.0)
        rz = dot(r, z)
        while active.any():
            if max_iterations is not None and total >= max_iterations:
                break
            total += 1
            q = prob.K(p, active)
            den = dot(p, q)
            valid = np.isfinite(den) & (den > 0) & np.isfinite(rz) & (rz > 0)
            failed = active & ~valid
            with np.errstate(divide="ignore", invalid="ignore"):
                alpha = np.where(active & valid, rz / np.where(valid, den, 1.0), 0.0)
            u = u + alpha[:, None] * p
            r = r - alpha[:, None] * q
            res2 = dot(r, r)
            finite = np.isfinite(res2)
            iterations = iterations + active.astype(np.int64)
            keep = active & valid & finite & (res2 > target2) & (iterations < iteration_cap)
            bad = bad | failed | (active & ~finite)
            active = keep
            z = prob.B(r)
            newrz = dot(r, z)
            with np.errstate(divide="ignore", invalid="ignore"):
                beta = np.where(active, newrz / np.where(rz != 0, rz, 1.0), 0.0)
            p = np.where(active[:, None], z + beta[:, None] * p, 0.0)
            rz = newrz
        u, r, absolute = certify(u)
        thr = np.sqrt(target2)
        ok = np.isfinite(absolute) & (absolute <= thr) & ~bad
        if max_iterations is not None and total >= max_iterations:
            break
        if ok.all() or restarts >= max_restarts or bad.any() or np.any(~ok & (iterations >= iteration_cap)):
            break
        restarts += 1
    thr = np.sqrt(target2)
    ok = np.isfinite(absolute) & (absolute <= thr) & ~bad
    infos = [SolveInfo(float(norm[j]), float(absolute[j]), float(thr[j]), int(iterations[j]),
                       float(absolute[j] / max(norm[j], 1e-300)), bool(ok[j]), restarts) for j in range(L)]
    return u, infos, not ok.all()


# ----------------------------------------------------------------------------- energies / C_H
def voigt_tensor(macro: np.ndarray) -> np.ndarray:
    m = macro
    return np.array([[m[0], m[5] / 2, m[4] / 2], [m[5] / 2, m[1], m[3] / 2], [m[4] / 2, m[3] / 2, m[2]]])


def affine(n: int, macros: np.ndarray) -> np.ndarray:
    """(L, 24) element-local affine displacement offsets/n . E^T (``backend.py:153-162``)."""
    off = local_offsets() / n
    return np.array([(off @ voigt_tensor(m).T).reshape(-1) for m in np.atleast_2d(macros)])


def energies(u: np.ndarray, aff: np.ndarray, n: int, lam: float, mu: float) -> np.ndarray:
    """e_l(el) = v^T Ke(C0) v / h^3, v = u_l(el) + A_l (``asg_scenarios_20261105/energy.cu:7-24``)."""
    ke = element_stiffness(n, lam, mu)
    v = _gather(_as_nodes(np.atleast_2d(u), n)) + aff[:, None, :]
    kv = v @ ke
    return (v * kv).sum(-1) * n ** 3


def effective_tensor(a: np.ndarray, u: np.ndarray, lam: float, mu: float, macros=None) -> np.ndarray:
    """6x6 homogenized tensor by polarization (``reproduction.py:166-176``)."""
    n = a.shape[0]
    macros = np.eye(6) if macros is None else macros
    aff = affine(n, macros)
    e = energies(u, aff, n, lam, mu)
    d = (e * a.reshape(1, -1)).mean(1)
    C = np.diag(d)
    for i in range(6):
        for j in range(i + 1, 6):
            pair = energies(u[i:i + 1] + u[j:j + 1], aff[i:i + 1] + aff[j:j + 1], n, lam, mu)
            q = (pair * a.reshape(1, -1)).mean()
            C[i, j] = C[j, i] = 0.5 * (q - d[i] - d[j])
    return C


def homogenize(a: np.ndarray, lam: float, mu: float, alpha: float, rtol: float = 1e-8, u0=None,
               macros=None, max_iterations: int | None = None, order: str = "a"):
    """One certified multi-load homogenization (all loads as parallel recurrences)."""
    macros = np.eye(6) if macros is None else np.atleast_2d(macros)
    prob = Problem(a, lam, mu, alpha)
    f = rhs(prob.a, macros, lam, mu)
    u, infos, raised = solve_batch(prob, f, u0, rtol, max_iterations=max_iterations, order=order)
    C = effective_tensor(prob.a, u, lam, mu, macros) if macros.shape[0] == 6 else None
    return dict(u=u, infos=infos, raised=raised, C=C, f=f)


# ----------------------------------------------------------------------------- generators
def baseline_density(n: int, seed: int, vf: float = 0.35, sigma_cells: float | None = None,
                     width: float = 0.1) -> np.ndarray:
    """Seeded N(0,1) noise -> periodic Gaussian (sigma=n/16) -> quantile threshold to ``vf``.

    The smooth threshold is rho = logistic((f - q_{1-vf}) / (width * std f)).
    """
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n, n, n))
    sig = n / 16.0 if sigma_cells is None else sigma_cells
    f = gaussian_filter(noise, sig, mode="wrap")
    q = np.quantile(f, 1.0 - vf)
    t = (f - q) / (width * f.std())
    return 1.0 / (1.0 + np.exp(-t))


def simp(rho: np.ndarray, emin: float, p: float = 3.0) -> np.ndarray:
    """E = Emin + rho^p (E0 - Emin), E0 = 1."""
    return emin + rho ** p * (1.0 - emin)


def study1_filter(x: np.ndarray) -> np.ndarray:
    """Periodic Gaussian, sigma = 0.9 n / 32 (``study.py:61``)."""
    from scipy.ndimage import gaussian_filter

    return gaussian_filter(x, 0.9 * x.shape[0] / 32, mode="wrap")


def study1_physical(x: np.ndarray, beta: float):
    """tanh projection at 0.5 (``study.py:64-67``)."""
    t = study1_filter(x)
    den = 2 * np.tanh(beta / 2)
    ph = (np.tanh(beta / 2) + np.tanh(beta * (t - 0.5))) / den
    dp = beta * (1 - np.tanh(beta * (t - 0.5)) ** 2) / den
    return ph, dp


def study1_material(ph: np.ndarray) -> np.ndarray:
    """SIMP eta=1e-4, p=3 (``study.py:70``)."""
    return 1e-4 + (1 - 1e-4) * ph ** 3


def study1_initial(n: int, seed: int) -> np.ndarray:
    """Twelve random cosine modes, volume-matched by 50 bisections (``study.py:73-88``)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*([(np.arange(n) + 0.5) / n] * 3), indexing="ij")
    fld = np.zeros((n, n, n))
    for _ in range(12):
        k = rng.integers(-2, 3, 3)
        if not np.any(k):
            k[0] = 1
        fld += rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + rng.uniform(0, 2 * np.pi))
    fld = 0.12 * fld / fld.std()
    lo, hi = -1.0, 1.0
    cand = None
    for _ in range(50):
        shift = (lo + hi) / 2
        cand = np.clip(0.3 + fld + shift, 0.01, 0.99)
        if study1_physical(cand, 1.0)[0].mean() > 0.3:
            hi = shift
        else:
            lo = shift
    return cand


def study1_state0(n: int, seed: int = 20261104) -> np.ndarray:
    """Study I design state 0: a = material(physical(initial(n, seed), 1)[0])."""
    return study1_material(study1_physical(study1_initial(n, seed), 1.0)[0])


def study1_oc(x, gradient, volume_gradient, beta, volume=0.3, move=0.1):
    """Study I OC with 45 bisections (``study.py:91-100``)."""
    lower = np.maximum(0.0, x - move)
    upper = np.minimum(1.0, x + move)
    ratio = np.maximum(gradient, 1e-30) / np.maximum(volume_gradient, 1e-30)
    lo, hi = 0.0, float(ratio.max()) * 1e4
    cand = x
    for _ in range(45):
        lam_ = (lo + hi) / 2
        cand = np.clip(x * np.sqrt(ratio / max(lam_, 1e-30)), lower, upper)
        if study1_physical(cand, beta)[0].mean() > volume:
            lo = lam_
        else:
            hi = lam_
    return cand


# Study II (paper) conventions -------------------------------------------------
def cone_stencil(rmin: float):
    """Offsets (dx,dy,dz) and weights rmin - |d| > 0 (``reproduction.py:38-45``)."""
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


def cone_filter(x: np.ndarray, rmin: float) -> np.ndarray:
    """Clipped (non-periodic) cone filter, unnormalised (``outer.cu:8-19``)."""
    n = x.shape[0]
    offs, ws = cone_stencil(rmin)
    out = np.zeros_like(x)
    for (dx, dy, dz), w in zip(offs, ws):
        src = np.zeros_like(x)
        zs = slice(max(0, dz), n + min(0, dz))
        zd = slice(max(0, -dz), n + min(0, -dz))
        ys = slice(max(0, dy), n + min(0, dy))
        yd = slice(max(0, -dy), n + min(0, -dy))
        xs = slice(max(0, dx), n + min(0, dx))
        xd = slice(max(0, -dx), n + min(0, -dx))
        src[zd, yd, xd] = x[zs, ys, xs]
        out += w * src
    return out


def paper_physical(t, hs, beta=4.0, eta=0.5, emin=1e-9):
    """tanh(beta, eta) projection + SIMP (``outer.cu:20-28``)."""
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    q = np.tanh(beta * (t / hs - eta))
    rho = (np.tanh(beta * eta) + q) / den
    return rho, beta * (1 - q * q) / den, emin + (1 - emin) * rho ** 3


def paper_local_energy(u, n, lam, mu, objective="shear", iteration=0):
    """Local objective density of the Study II objectives (``reproduction.py:153-164``).

    ``u`` holds the six Voigt-load solutions. The hydrostatic solution is u0 + u1 + u2 by linearity.
    Returns (local (N,), per-load energies (6, N)).
    """
    e = energies(u, affine(n, np.eye(6)), n, lam, mu)
    if objective == "shear":
        return -e[3:].sum(0), e
    hydro = energies(u[:3].sum(0, keepdims=True), affine(n, [[1.0, 1.0, 1.0, 0.0, 0.0, 0.0]]), n, lam, mu)[0]
    if objective == "bulk":
        return -hydro, e
    if objective == "auxetic":
        return hydro - (1 + 0.8 ** iteration) * e[:3].sum(0), e
    raise ValueError(objective)


def paper_sensitivity(energy, ph, dp, hs, rmin, emin=1e-9):
    """Filtered objective and volume sensitivities d/dx of mean(local * a) and of sum(rho)
    (``reproduction.py:91-94``; the check of ``asg_sctop_reproduction_20261105/verify.py:60-61``)."""
    n = ph.shape[0]
    g = cone_filter(dp * (3 * (1 - emin) * ph * ph) * energy / hs, rmin) / n ** 3
    return g, cone_filter(dp / hs, rmin)


def paper_oc(x, energy, ph, dp, hs, rmin, volume, beta=4.0, eta=0.5, emin=1e-9, move=0.1,
             exponent=0.3, floor=0.001, max_steps=180):
    """Damped OC with MATLAB-style bisection stop (``reproduction.py:91-104``, ``outer.cu:29-39``).

    ``energy`` is the local objective density (negative for stiffness maximisation).
    Returns (new, steps, change).
    """
    g, dv = paper_sensitivity(energy, ph, dp, hs, rmin, emin)
    ratio = -g / dv
    lo, hi, flag, steps = 0.0, 1e9, 1.0, 0
    new = x.copy()
    for _ in range(max_steps):
        if flag == 0.0:
            break
        mid = 0.5 * (lo + hi)
        v = x * np.maximum(1e-10, ratio / mid) ** exponent
        new = np.maximum(floor, np.maximum(x - move, np.minimum(1.0, np.minimum(x + move, v))))
        t = cone_filter(new, rmin)
        rho, _, _ = paper_physical(t, hs, beta, eta, emin)
        vol = rho.mean()
        mid = 0.5 * (lo + hi)
        if vol > volume:
            lo = mid
        else:
            hi = mid
        steps += 1
        flag = 1.0 if ((hi - lo) / (hi + lo) > 1e-4 and hi > 1e-40) else 0.0
    return new, steps, float(np.abs(new - x).max())


# ----------------------------------------------------------------------------- alpha selectors
def law_features(a: np.ndarray) -> np.ndarray:
    """(area, jump, contrast, complexity) in FP32 (``solver/experiments/global_alpha_compact_law/law.py:10-19``)."""
    ell = np.log(a.astype(np.float32))
    lo, hi = ell.min(), ell.max()
    span = np.float32(hi - lo)
    q = (ell - lo) / max(span, np.float32(1e-12))
    s1 = s2 = act = np.float32(0)
    for axis in range(3):
        d = np.abs(np.roll(q, -1, axis) - q)
        s1 = s1 + d.mean(dtype=np.float32)
        s2 = s2 + (d * d).mean(dtype=np.float32)
        act = act + (d > 1e-6).astype(np.float32).mean(dtype=np.float32)
    area = act / np.float32(3)
    jump = s2 / max(s1, np.float32(1e-20))
    return np.array([area, jump, span / np.float32(np.log(10000.0)), area * a.shape[0]], dtype=np.float32)


def compact8_alpha(a: np.ndarray, quantize: bool = False) -> float:
    """Compact law with exponent 8 and the 0.375 cut-off (``asg_density_selector_20261105/run.py:60-66``)."""
    area, jump, contrast, complexity = (float(v) for v in law_features(a))
    if not (complexity > 1e-12 and contrast > 1e-12):
        return 0.0
    v = 1.0 - 0.75 * np.sqrt(max(area * jump, 0.0)) / np.sqrt(max(contrast, 1e-30)) - (2.5 / max(complexity, 1e-30)) ** 8
    v = min(1.0, max(0.0, v))
    v = 0.0 if v < 0.375 else v
    return float(np.floor(16 * v + 0.5) / 16) if quantize else v


def _contrast_base(a, anchors):
    s = min(9.0, max(0.0, float(np.log10(a.max() / a.min()))))
    b4, b6, b9 = anchors
    if s < 4:
        return s, b4 * s / 4
    if s < 6:
        return s, b4 + (b6 - b4) * (s - 4) / 2
    return s, b6 + (b9 - b6) * (s - 6) / 3


def contrast_alpha(a: np.ndarray, anchors=(0.5625, 0.6875, 0.8125)) -> float:
    """Contrast model rounded to sixteenths (``asg_density_selector_20261105/run.py:27-33``)."""
    s, base = _contrast_base(a, anchors)
    return float(np.floor(min(1.0, max(0.0, base)) * 16 + 0.5) / 16) if s > 1e-12 else 0.0


def gray_alpha(a: np.ndarray, rho: np.ndarray, anchors=(0.5625, 0.75, 0.8125), gamma=0.075,
               g_ref=0.3739899920170806) -> float:
    """Contrast model shifted by the grayness of rho (``asg_density_selector_20261105/run.py:36-43``)."""
    s, base = _contrast_base(a, anchors)
    v = rho.mean()
    g = min(1.0, max(0.0, float((v - (rho * rho).mean()) / (v * (1 - v) + 1e-12))))
    value = base + gamma * (g_ref - g)
    return float(np.floor(min(1.0, max(0.0, value)) * 16 + 0.5) / 16) if s > 1e-12 else 0.0
