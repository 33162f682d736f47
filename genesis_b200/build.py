"""Builds the sm_100a shared library ``libgenesis_gpu.so`` in-tree.

Run ``python -m genesis_b200.build`` (or call :func:`build`).  The library is
plain CUDA C++ with a C ABI (``include/genesis_gpu.h``); nvcc cross-compiles
it without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
LIB = PKG / "libgenesis_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources() -> list[Path]:
    return sorted(SRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(SRC.glob("*.cuh")) + [ROOT / "include" / "genesis_gpu.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles every ``csrc/*.cu`` into ``libgenesis_gpu.so`` for sm_100a."""
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, f"-I{ROOT / 'include'}", f"-I{SRC}"]
    cmd += list(extra or [])
    cmd += [str(s) for s in sources()]
    cmd += ["-o", str(LIB) + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
