"""In-tree build of the CUDA library (``libhnsw_b200.so``) for sm_100a with nvcc.

The library is a plain shared object with a C ABI (``include/hnsw_b200.h``); it links only the
CUDA runtime, so it loads through ctypes with no PyTorch types across the boundary.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = sorted((PKG / "csrc").glob("*.cu")) + sorted((PKG / "csrc").glob("*.cpp"))  # .cpp: host only
OUT = PKG / "libhnsw_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).is_file():
            return cand
    raise FileNotFoundError("nvcc not found")


def needs_build() -> bool:
    if not OUT.is_file():
        return True
    stamp = OUT.stat().st_mtime
    deps = list(SOURCES) + list((PKG / "csrc").glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(p.stat().st_mtime > stamp for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every ``csrc/*.cu`` and ``csrc/*.cpp`` into ``libhnsw_b200.so`` (skipped when up to
    date)."""
    if not force and not needs_build():
        return OUT
    cmd = [
        nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-shared", f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}",
        "-o", str(OUT), *map(str, SOURCES),
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
