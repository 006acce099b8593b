"""Build recipe of libglu_gfix.so (sm_100a), in tree under glu_b200/_lib/.

    python -m glu_b200.build          # or build() from Python

nvcc cross-compiles for sm_100a without a GPU.  The library is plain
CUDA C++ with a C ABI (include/glu_gfix.h): no torch types.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libglu_gfix.so"
SOURCES = ["gfix.cu", "glu_abi.cu", "noalloc.cu", "nersc.cu", "cuts.cu", "update.cu"]
HEADERS = ["su3.cuh", "fft.cuh", "fft_pass.cuh", "fft_ct.cuh", "kernels.cuh", "extra_kernels.cuh",
           "coulomb.cuh", "glu_compat.h", "su3_log.cuh", "drop_in.h"]

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
    """Compile every translation unit to an object (in parallel: the units
    share no device code), then link the shared library."""
    if not force and not stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = LIB_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    objs = [obj_dir / (s.stem + ".o") for s in srcs]
    cmds = [[_nvcc(), *compile_flags, "-c", "-o", str(o), str(s)]
            for s, o in zip(srcs, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, cwd=str(CSRC)), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
            "-Xcompiler", "-fopenmp", "-o", str(LIB), *[str(o) for o in objs],
            "-lgomp"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True, cwd=str(CSRC))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
