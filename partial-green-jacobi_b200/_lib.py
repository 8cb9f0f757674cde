"""ctypes binding of libpgj.so (the C ABI declared in include/pgj.h).

The shared library is built in-tree by ``build.py`` for sm_100a. There is no fallback: if the
library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpgj.so"

PGJ_OK = 0
PGJ_ERR_ARGUMENT = 1
PGJ_ERR_UNSUPPORTED = 2
PGJ_ERR_LAUNCH = 3
PGJ_ERR_NONFINITE = 4
PGJ_ERR_ITERATION_CAP = 5
PGJ_ERR_CERTIFICATION = 6
PGJ_ERR_TIMEOUT = 7
PGJ_ERR_WORKSPACE = 8
PGJ_FP64 = 0
PGJ_FP32 = 1

vp = C.c_void_p
i32 = C.c_int32
f64 = C.c_double
sz = C.c_size_t


class LoadInfo(C.Structure):
    _fields_ = [("rhs_norm", f64), ("absolute_residual", f64), ("threshold", f64), ("relative_residual", f64),
                ("iterations", i32), ("converged", i32), ("restarts", i32), ("bad", i32)]

    def as_dict(self) -> dict:
        return dict(rhs_norm=self.rhs_norm, absolute_residual=self.absolute_residual, threshold=self.threshold,
                    iterations=int(self.iterations), relative_residual=self.relative_residual,
                    converged=bool(self.converged), restarts=int(self.restarts))


# name -> (restype, argtypes)
SIGNATURES = {
    "pgj_version": (C.c_int, []),
    "pgj_status_string": (C.c_char_p, [C.c_int]),
    "pgj_last_cuda_error": (C.c_int, []),
    "pgj_workspace_bytes": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(sz)]),
    "pgj_ctx_create": (C.c_int, [C.c_int, C.c_int, C.c_int, f64, f64, vp, sz, vp, C.POINTER(vp)]),
    "pgj_ctx_destroy": (C.c_int, [vp]),
    "pgj_workspace_bytes_batch": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(sz)]),
    "pgj_ctx_create_batch": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, f64, f64, vp, sz, vp, C.POINTER(vp)]),
    "pgj_ctx_designs": (C.c_int, [vp]),
    "pgj_set_material_at": (C.c_int, [vp, C.c_int, vp, vp]),
    "pgj_set_alpha_at": (C.c_int, [vp, C.c_int, f64, vp]),
    "pgj_effective_tensor_at": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "pgj_ctx_solutions": (vp, [vp]),
    "pgj_ctx_scale": (vp, [vp]),
    "pgj_ctx_material": (vp, [vp]),
    "pgj_set_material": (C.c_int, [vp, vp, vp]),
    "pgj_set_alpha": (C.c_int, [vp, f64, vp]),
    "pgj_apply": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "pgj_apply_f32": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "pgj_rhs": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "pgj_precondition": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "pgj_green_symbol": (C.c_int, [C.c_int, f64, f64, vp, vp]),
    "pgj_solve": (C.c_int, [vp, C.c_int, vp, f64, vp, C.POINTER(LoadInfo), vp]),
    "pgj_solve_async": (C.c_int, [vp, C.c_int, vp, f64, vp, vp]),
    "pgj_solve_wait": (C.c_int, [vp, C.POINTER(LoadInfo), vp]),
    "pgj_set_inner_rtol": (C.c_int, [vp, f64]),
    "pgj_set_mixed_mode": (C.c_int, [vp, C.c_int, f64]),
    "pgj_set_mixed_operator": (C.c_int, [vp, C.c_int]),
    "pgj_set_iteration_cap": (C.c_int, [vp, C.c_int]),
    "pgj_set_flexible_beta": (C.c_int, [vp, C.c_int]),
    "pgj_iteration_cap": (C.c_int, [vp]),
    "pgj_last_refinements": (C.c_int, [vp]),
    "pgj_last_launches": (C.c_longlong, [vp]),
    "pgj_selftest_wait_timeout": (C.c_int, [vp, C.c_int, vp]),
    "pgj_fused_iteration": (C.c_int, [vp]),
    "pgj_tile_shapes": (C.c_int, [vp, C.POINTER(C.c_int)]),
    "pgj_tile_config": (C.c_int, [vp, C.POINTER(C.c_int)]),
    "pgj_set_fused_iteration": (C.c_int, [vp, C.c_int]),
    "pgj_profile_iteration": (C.c_int, [vp, C.c_int, vp, C.c_int, vp, vp, vp]),
    "pgj_energies": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "pgj_effective_tensor": (C.c_int, [vp, vp, vp, vp]),
    "pgj_effective_tensor_noalloc": (C.c_int, [C.c_int, f64, f64, vp, vp, vp, vp]),
    "pgj_cone_filter": (C.c_int, [C.c_int, vp, vp, C.c_int, vp, vp, vp]),
    "pgj_paper_project": (C.c_int, [C.c_int, vp, vp, f64, f64, f64, vp, vp, vp, vp]),
    "pgj_paper_oc": (C.c_int, [C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, vp, f64, f64, f64, f64, f64, f64, f64,
                               vp, vp, C.POINTER(C.c_int), C.POINTER(f64), vp]),
    "pgj_gaussian_filter": (C.c_int, [C.c_int, vp, C.c_int, vp, vp, vp, vp]),
    "pgj_study1_project": (C.c_int, [C.c_int, vp, f64, vp, vp, vp, vp]),
    "pgj_study1_oc": (C.c_int, [C.c_int, vp, C.c_int, vp, vp, vp, vp, f64, f64, f64, vp, vp, C.POINTER(f64), vp]),
}


class PGJError(RuntimeError):
    def __init__(self, status: int, where: str, lib=None):
        msg = lib.pgj_status_string(status).decode() if lib is not None else f"status {status}"
        cuda = lib.pgj_last_cuda_error() if lib is not None else 0
        super().__init__(f"{where}: {msg}" + (f" (cuda error {cuda})" if status == PGJ_ERR_LAUNCH else ""))
        self.status = status


@lru_cache(None)
def lib() -> C.CDLL:
    if not LIB_PATH.exists():
        raise RuntimeError(f"libpgj.so not built at {LIB_PATH}; run `python partial-green-jacobi_b200/build.py` "
                           "(the CUDA extension is required: there is no CPU fallback)")
    handle = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


def check(status: int, where: str) -> None:
    if status != PGJ_OK:
        raise PGJError(status, where, lib())


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)
