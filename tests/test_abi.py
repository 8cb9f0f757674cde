"""The C ABI library loads without a GPU and exports every function include/pgj.h declares."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "pgj.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgj_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_surface():
    names = declared_functions()
    for required in ("pgj_ctx_create", "pgj_apply", "pgj_rhs", "pgj_precondition", "pgj_solve",
                     "pgj_effective_tensor", "pgj_paper_oc", "pgj_study1_oc"):
        assert required in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(pkg):
    assert set(declared_functions()) == set(pkg._lib.exported_symbols())


def test_status_strings_and_argument_errors_without_gpu(pkg):
    lib = pkg._lib.lib()
    assert lib.pgj_status_string(6) == b"true residual certification failed"
    nb = ctypes.c_size_t()
    assert lib.pgj_workspace_bytes(64, 6, 0, ctypes.byref(nb)) == 0 and nb.value > 6 * 3 * 64 ** 3 * 8
    assert lib.pgj_workspace_bytes(17, 6, 0, ctypes.byref(nb)) == 2  # odd / prime edge: unsupported
    assert lib.pgj_workspace_bytes(64, 0, 0, ctypes.byref(nb)) == 1
    assert lib.pgj_workspace_bytes(64, 6, 7, ctypes.byref(nb)) == 1
    assert lib.pgj_ctx_create(64, 6, 0, 1.0, 1.0, None, 0, None, ctypes.byref(ctypes.c_void_p())) == 8


def test_product_path_has_no_oracle_import():
    pkg_dir = ROOT / "partial-green-jacobi_b200"
    for p in pkg_dir.glob("*.py"):
        assert "pgj_oracle" not in p.read_text(), p
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\S+)", p.read_text(), flags=re.M), p


def test_package_modules_do_not_shadow_the_standard_library():
    """Scripts run from the package directory (build.py, profile_iteration.py, the drivers) put it
    first on sys.path, so no module there may share a standard-library name."""
    import sys
    from pathlib import Path

    pkg_dir = Path(__file__).resolve().parents[1] / "partial-green-jacobi_b200"
    names = {p.stem for p in pkg_dir.glob("*.py")}
    assert not names & set(sys.stdlib_module_names), names & set(sys.stdlib_module_names)
