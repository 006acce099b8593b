"""The C-ABI library: builds, loads, and exports every declared symbol.

No compute call is made here (no GPU needed)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    txt = (ROOT / "include" / "glu_gfix.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)
    skip = {"extern", "sizeof", "if", "defined"}
    return sorted({n for n in names if n not in skip})


def test_header_declares_the_glu_entry_points():
    decl = declared_functions()
    for n in ("FACG", "FASD", "Landau", "Coulomb", "Coulomb_FA",
              "FOURIER_ACCELERATE3", "FOURIER_ACCELERATE2"):
        assert n in decl


def test_library_loads_and_exports_every_declared_symbol():
    from glu_b200 import _lib, build
    try:
        build.build()
    except Exception as e:  # nvcc missing
        pytest.skip(f"cannot build: {e}")
    lib = _lib.load()
    for n in declared_functions():
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) == set(declared_functions())


def test_missing_library_fails_loudly(tmp_path):
    from glu_b200 import _lib
    with pytest.raises(_lib.GfixError):
        _lib.load(tmp_path / "nope.so") if _lib._lib is None else \
            (_ for _ in ()).throw(_lib.GfixError("already loaded"))
