"""Shared pytest setup.

Markers: ``gpu`` for tests that need a B200 (run with ``-m gpu``); the rest
run on the CPU.  The CPU checkers in oracle/ are built on first use.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a)")


def _ensure_oracle():
    from oracle import oracle as O
    if not O.ORACLE_SO.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"],
                       check=True, stdout=subprocess.DEVNULL)
    return O


@pytest.fixture(scope="session")
def oracle():
    O = _ensure_oracle()
    return O.Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference compiled from its sources; skipped where absent."""
    from oracle import oracle as O
    if not O.REF_SO.exists():
        pytest.skip("reference build (oracle/_ref) not present")
    return O.Reference()


@pytest.fixture(scope="session")
def lat400():
    return dict(np.load(GOLDEN / "lat400.npz"))


@pytest.fixture(scope="session")
def hb8():
    return dict(np.load(GOLDEN / "hb8.npz"))


@pytest.fixture(scope="session")
def headline_config():
    """The first configuration of the 32^3x64 Landau benchmark (GPU tests
    only): beta 6.0, 1000 heatbath + 4 over-relaxation iterations from the
    unit start, seed 2, generated on the GPU."""
    from glu_b200.workload import heatbath_config
    return heatbath_config((32, 32, 32, 64), seed=2, iterations=1000, beta=6.0, n_or=4)
