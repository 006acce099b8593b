"""Argument errors of the C-ABI entry points are reported before any device work.

The solvers (gfix_landau, gfix_coulomb and their _device forms,
gfix_landau_sequence), the
allocation-free theta/functional, the NERSC codec, the gluon-propagator
measurement and the heatbath generator validate their dimensions, parameters
and pointers first: a bad call returns -1 with a message in the matching
*_error() string and touches no CUDA state, so these run without a GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from glu_b200 import _lib
from glu_b200._lib import GfixParams, GfixResult


@pytest.fixture(scope="module")
def lib():
    from glu_b200 import build
    try:
        build.build()
    except Exception as e:  # nvcc missing
        pytest.skip(f"cannot build: {e}")
    return _lib.load()


def _params(**kw):
    p = GfixParams()
    p.gf_alpha, p.accuracy, p.max_iters = 0.08, 1e-14, 1000
    p.algo, p.sd_fixed_step, p.precision, p.switch_theta = 0, 0, 0, 1e-9
    p.traj_cap = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


LINKS = np.zeros(2 * 2 * 2 * 2 * 4 * 18)


def _call(lib, fn, dims, p, links=LINKS):
    cd = (C.c_size_t * 4)(*dims)
    ptr = None if links is None else links.ctypes.data
    r = GfixResult()
    if fn.startswith("gfix_coulomb"):
        rc = getattr(lib, fn)(ptr, cd, C.byref(p) if p is not None else None,
                              C.byref(r), None, None)
    else:
        rc = getattr(lib, fn)(ptr, cd, C.byref(p) if p is not None else None, C.byref(r))
    return rc, lib.gfix_last_error().decode()


FNS = ["gfix_landau", "gfix_landau_device", "gfix_coulomb", "gfix_coulomb_device"]


@pytest.mark.parametrize("fn", FNS)
@pytest.mark.parametrize("dims, kw, msg", [
    ((2, 2, 1, 2), {}, "extent 1 of dimension 2 below 2"),
    ((0, 2, 2, 2), {}, "extent 0 of dimension 0 below 2"),
    ((2, 2, 2, 2), {"algo": 7}, "unknown algo 7"),
    ((2, 2, 2, 2), {"precision": 5}, "unknown precision 5"),
    ((2, 2, 2, 2), {"traj_cap": 10}, "traj_cap without traj_theta"),
], ids=["extent1", "extent0", "algo", "precision", "traj"])
def test_bad_arguments_rejected(lib, fn, dims, kw, msg):
    rc, err = _call(lib, fn, dims, _params(**kw))
    assert rc == -1
    assert msg in err


@pytest.mark.parametrize("fn", FNS)
def test_null_links_and_params_rejected(lib, fn):
    rc, err = _call(lib, fn, (2, 2, 2, 2), _params(), links=None)
    assert rc == -1 and "null links" in err
    rc, err = _call(lib, fn, (2, 2, 2, 2), None)
    assert rc == -1 and "null dims or params" in err


def test_sequence_arguments_rejected(lib):
    """gfix_landau_sequence: the parameters as gfix_landau's, then the
    pointer array and every configuration's pointer; n = 0 is a no-op."""
    cd = (C.c_size_t * 4)(2, 2, 2, 2)
    r = (GfixResult * 2)()
    assert lib.gfix_landau_sequence(None, 0, cd, C.byref(_params()), r) == 0
    assert lib.gfix_landau_sequence(None, 2, cd, C.byref(_params(algo=7)), r) == -1
    assert "unknown algo 7" in lib.gfix_last_error().decode()
    assert lib.gfix_landau_sequence(None, 2, cd, C.byref(_params()), r) == -1
    assert "null argument" in lib.gfix_last_error().decode()
    ptrs = (C.c_void_p * 2)(LINKS.ctypes.data, None)
    assert lib.gfix_landau_sequence(ptrs, 2, cd, C.byref(_params()), r) == -1
    assert "null links of configuration 1" in lib.gfix_last_error().decode()


def test_null_batch_rejected(lib):
    assert lib.gfix_batch_run(None) == -1
    assert "null batch" in lib.gfix_last_error().decode()


@pytest.mark.parametrize("dims, msg", [
    ((256, 256, 256, 2), "at most 16777216 sites"),
    # a volume that wraps around 2^64 to exactly 2^24 sites
    (((1 << 40) + 1, 1 << 22, 2, 2), "at most 16777216 sites"),
    ((2, 1, 2, 2), "every extent must be at least 2"),
], ids=["too-large", "wraps", "extent1"])
def test_noalloc_limits_rejected(lib, dims, msg):
    # rejected before the pointers are used, so stand-in addresses serve
    cd = (C.c_size_t * 4)(*dims)
    assert lib.gfix_theta_functional_noalloc(C.c_void_p(256), cd, C.c_void_p(512),
                                             None) == -1
    assert msg in lib.gfix_noalloc_error().decode()


def test_noalloc_null_rejected(lib):
    cd = (C.c_size_t * 4)(4, 4, 4, 4)
    assert lib.gfix_theta_functional_noalloc(None, cd, C.c_void_p(512), None) == -1
    assert "null argument" in lib.gfix_noalloc_error().decode()


def test_noalloc_error_is_per_thread(lib):
    """The message buffer is thread-local: a failure on another thread does
    not overwrite this thread's message."""
    import threading
    cd = (C.c_size_t * 4)(4, 4, 4, 4)
    assert lib.gfix_theta_functional_noalloc(None, cd, C.c_void_p(512), None) == -1
    other = []

    def run():
        big = (C.c_size_t * 4)(256, 256, 256, 2)
        lib.gfix_theta_functional_noalloc(C.c_void_p(256), big, C.c_void_p(512), None)
        other.append(lib.gfix_noalloc_error().decode())

    t = threading.Thread(target=run)
    t.start()
    t.join()
    assert "16777216" in other[0]
    assert "null argument" in lib.gfix_noalloc_error().decode()


@pytest.mark.parametrize("fn", ["gfix_nersc_decode", "gfix_nersc_encode"])
@pytest.mark.parametrize("dims, nreal, nbytes, msg", [
    ((2, 2, 2, 2), 10, 8, "reals per link must be 12 or 18"),
    ((2, 2, 2, 2), 18, 2, "bytes per real must be 8 or 4"),
    ((2, 0, 2, 2), 18, 8, "zero extent"),
], ids=["nreal", "bytes", "extent"])
def test_nersc_bad_arguments_rejected(lib, fn, dims, nreal, nbytes, msg):
    cd = (C.c_size_t * 4)(*dims)
    buf = np.zeros(2 * 2 * 2 * 2 * 4 * 18)
    assert getattr(lib, fn)(buf.ctypes.data, cd, nreal, nbytes, 1, buf.ctypes.data,
                            None) == -1
    assert msg in lib.gfix_nersc_error().decode()


@pytest.mark.parametrize("fn", ["gfix_nersc_decode", "gfix_nersc_encode"])
def test_nersc_null_rejected(lib, fn):
    cd = (C.c_size_t * 4)(2, 2, 2, 2)
    assert getattr(lib, fn)(None, cd, 18, 8, 1, None, None) == -1
    assert "null payload or links" in lib.gfix_nersc_error().decode()


@pytest.mark.parametrize("fn", ["gfix_heatbath", "gfix_heatbath_device"])
def test_heatbath_bad_arguments_rejected(lib, fn):
    f = getattr(lib, fn)
    # the draughtboard update needs even extents
    cd = (C.c_size_t * 4)(4, 4, 3, 4)
    assert f(LINKS.ctypes.data, cd, 6.0, 1, 4, 1, 0, None) == -1
    assert "needs even extents" in lib.gfix_update_error().decode()
    assert f(None, cd, 6.0, 1, 4, 1, 0, None) == -1
    assert "null links" in lib.gfix_update_error().decode()


@pytest.mark.parametrize("fn", ["gfix_cuts_measure", "gfix_cuts_measure_device"])
@pytest.mark.parametrize("kw, msg", [
    ({"dir": 1}, "cut mode 1 not supported"),
    ({"type": 9}, "momentum cut type 9 unknown"),
    ({"definition": 7}, "field definition 7 unknown"),
], ids=["nonexceptional", "type", "definition"])
def test_cuts_bad_arguments_rejected(lib, fn, kw, msg):
    from glu_b200._lib import GfixCutInfo
    ci = GfixCutInfo(dir=6, type=2, max_mom=4, definition=0, angle=60, cyl_width=2.0)
    for k, v in kw.items():
        setattr(ci, k, v)
    cd = (C.c_size_t * 4)(2, 2, 2, 2)
    out = np.zeros(16)
    f = getattr(lib, fn)
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    assert f(LINKS.ctypes.data, cd, C.byref(ci), 1, ptr(out), ptr(out), ptr(out)) == -1
    assert msg in lib.gfix_cuts_error().decode()
    assert f(None, cd, C.byref(ci), 1, ptr(out), ptr(out), ptr(out)) == -1
    assert "null links" in lib.gfix_cuts_error().decode()


def test_python_mirror_raises_the_library_message(lib):
    # the host mirror checks shapes itself and raises the C library's
    # message for what the library rejects
    from glu_b200 import gfix
    U = np.zeros((2 * 2 * 1 * 2, 4, 3, 3), complex)
    with pytest.raises(_lib.GfixError, match="extent 1 of dimension 2 below 2"):
        gfix.landau_fix(U, (2, 2, 1, 2))
    with pytest.raises(_lib.GfixError, match="extent 1 of dimension 2 below 2"):
        gfix.coulomb_fix(U, (2, 2, 1, 2))
    with pytest.raises(ValueError, match="dims must be"):
        gfix.landau_fix(U, (2, 2, 2))
    with pytest.raises(ValueError, match="sites"):
        gfix.landau_fix(U, (2, 2, 2, 2))
