"""Build recipe of libglu_gfix.so (sm_100a), in tree under glu_b200/_lib/.

    python -m glu_b200.build          # or build() from Python

nvcc cross-compiles for sm_100a without a GPU.  The library is plain
CUDA C++ with a C ABI (include/glu_gfix.h): no torch types.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libglu_gfix.so"
SOURCES = ["gfix.cu", "glu_abi.cu", "noalloc.cu", "nersc.cu", "cuts.cu", "update.cu"]
HEADERS = ["su3.cuh", "fft.cuh", "fft_pass.cuh", "fft_ct.cuh", "kernels.cuh", "extra_kernels.cuh",
           "coulomb.cuh", "glu_compat.h", "su3_log.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
    "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    return "nvcc"


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS]
    deps.append(ROOT / "include" / "glu_gfix.h")
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", str(LIB),
           *[str(CSRC / s) for s in SOURCES if (CSRC / s).exists()], "-lgomp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
