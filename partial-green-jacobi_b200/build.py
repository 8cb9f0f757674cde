"""Build libpgj.so in-tree for sm_100a with nvcc (no JIT, no torch headers).

    python partial-green-jacobi_b200/build.py [--verbose]

The library is a plain C-ABI shared object; the Python package binds it with ctypes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libpgj.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpgj")
    return path


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not OUT.exists():
        return True
    stamp = OUT.stat().st_mtime
    deps = (list(sources()) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc"))
            + [HERE.parent / "include/pgj.h"])
    return any(p.stat().st_mtime > stamp for p in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", str(HERE.parent / "include"), "-o", str(tmp), *map(str, sources())]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    jobs = os.environ.get("PGJ_NVCC_THREADS", "8")
    cmd[1:1] = ["--threads", jobs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
