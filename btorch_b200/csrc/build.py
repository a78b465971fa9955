"""Build the C-ABI shared library libbtorch_b200.so for sm_100a with nvcc.

Usage: python -m btorch_b200.csrc.build   (or called from __graft_entry__.build)
The library lands next to this package (btorch_b200/_lib/) so it travels with
the source tree; it links the CUDA runtime statically and exports only the
extern "C" symbols declared in include/btorch_b200.h.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent
ROOT = PKG.parent
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libbtorch_b200.so"
SOURCES = ["layout.cpp", "spmv.cu", "neuron.cu", "engine.cu", "tile.cu", "cluster.cu", "raster.cu"]
HEADERS = ["common.cuh", "neuron.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda_home) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _stale() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "btorch_b200.h"]
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        nvcc(),
        *ARCH,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC,-fvisibility=hidden",
        "-shared",
        "-cudart",
        "static",
        "-o",
        str(tmp),
        *[str(CSRC / s) for s in SOURCES],
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
