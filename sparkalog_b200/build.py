"""Builds the in-tree CUDA library ``sparkalog_b200/lib/libsparkalog_b200.so``.

The library is compiled for sm_100a only, with nvcc called directly (no
torch JIT cache), so the built ``.so`` sits inside the repository tree and
travels with it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR / "csrc"
LIB_DIR = PACKAGE_DIR / "lib"
LIB_PATH = LIB_DIR / "libsparkalog_b200.so"
INCLUDE_DIR = PACKAGE_DIR.parent / "include"

SOURCES = [
    "abi_operators.cu",
    "abi_no_alloc.cu",
    "engine.cu",
]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda_home) / "bin" / "nvcc"
    if candidate.exists():
        return str(candidate)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every source to an object and links the shared library."""
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = PACKAGE_DIR / "_build"
    obj_dir.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE_DIR.glob("*.h"))
    objects = []
    for src in SOURCES:
        src_path = CSRC / src
        obj = obj_dir / (src_path.stem + ".o")
        objects.append(obj)
        if force or _stale(obj, [src_path, *headers]):
            cmd = [nvcc(), *NVCC_FLAGS, "-I", str(CSRC), "-I", str(INCLUDE_DIR), "-c", str(src_path), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB_PATH, objects):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB_PATH),
               *map(str, objects), "-lcuda"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
