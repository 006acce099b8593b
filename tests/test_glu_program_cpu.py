"""Host-side behaviour of the GLU-named entry points, without a GPU.

Inside GLU's own program (linked against the library) a thread started at
load time creates the device context and pins the staging chunks; any other
process -- Python loading the library, for instance -- is left alone.  With
no usable device, GLU's program still runs: Landau() reports why it cannot
stage the links on GLU's error stream and returns GLU_FAILURE, which GLU's
program survives as it does any failed fix.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import pytest

from conftest import GOLDEN, ROOT
from glu_structs import GLU_INPUT

LIB = ROOT / "glu_b200" / "_lib" / "libglu_gfix.so"


def _no_device() -> bool:
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


def test_a_python_process_is_not_a_glu_program():
    """Loading the library from Python starts no warm-up thread and leaves
    the module-loading mode of the process alone."""
    if not LIB.exists():
        pytest.skip("library not built")
    code = ("import ctypes as C\n"
            f"C.CDLL({str(LIB)!r})\n"
            "libc = C.CDLL(None)\n"
            "libc.getenv.restype = C.c_char_p\n"
            "print(libc.getenv(b'CUDA_MODULE_LOADING'))\n")
    env = {k: v for k, v in os.environ.items() if k != "CUDA_MODULE_LOADING"}
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env=env, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == "None"


@pytest.mark.skipif(not _no_device(), reason="a CUDA device is present")
def test_relinked_program_without_a_device(tmp_path):
    gpu = ROOT / "oracle" / "_ref" / "glu_gpu"
    if not gpu.exists():
        pytest.skip("oracle/_ref/glu_gpu not built")
    inp = tmp_path / "in"
    inp.write_text(GLU_INPUT.format(d0=4, d1=4, d2=4, d3=8, gftype="LANDAU", tune=0.08,
                                    max_iters=650))
    p = subprocess.run([str(gpu), "-i", str(inp), "-c", str(GOLDEN / "lat400.nersc")],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert p.returncode == 0
    assert "[GF] allocation of the GPU staging chunks failed" in p.stderr
    # GLU read the configuration and reached its gauge-fixing wrapper
    assert "[GF] Landau gauge, accuracy of 1e-14" in p.stdout
