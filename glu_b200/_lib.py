"""ctypes binding of libglu_gfix.so (the C ABI in include/glu_gfix.h).

There is no CPU fallback: if the library is missing or cannot be loaded,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .build import LIB

_dp = C.POINTER(C.c_double)
_szp = C.POINTER(C.c_size_t)


class GfixParams(C.Structure):
    _fields_ = [("gf_alpha", C.c_double), ("accuracy", C.c_double),
                ("max_iters", C.c_size_t), ("algo", C.c_int),
                ("sd_fixed_step", C.c_int), ("precision", C.c_int),
                ("switch_theta", C.c_double), ("traj_theta", _dp),
                ("traj_func", _dp), ("traj_cap", C.c_size_t),
                ("max_restarts", C.c_int), ("restart_seed", C.c_uint64),
                ("luxury_copies", C.c_int), ("luxury_best", C.c_int)]


class GfixCutInfo(C.Structure):
    _fields_ = [("dir", C.c_int), ("type", C.c_int), ("max_mom", C.c_size_t),
                ("definition", C.c_int), ("angle", C.c_size_t),
                ("cyl_width", C.c_double)]


class GfixResult(C.Structure):
    _fields_ = [("iters", C.c_size_t), ("iters_fp32", C.c_size_t),
                ("theta", C.c_double), ("traj_len", C.c_size_t),
                ("gpu_ms", C.c_double), ("restarts", C.c_int)]


# every symbol include/glu_gfix.h declares
EXPORTS = ("FACG", "FASD", "FOURIER_ACCELERATE3", "Landau", "Coulomb",
           "Coulomb_FA", "FOURIER_ACCELERATE2", "cuts_struct", "gfix_landau",
           "gfix_landau_sequence", "gfix_landau_device", "gfix_landau_driver", "gfix_coulomb",
           "gfix_coulomb_device", "gfix_coulomb_driver",
           "gfix_observables", "gfix_reunit", "gfix_fourier_accelerate",
           "gfix_profile_landau", "gfix_profile_coulomb",
           "gfix_theta_functional_noalloc", "gfix_batch_create",
           "gfix_batch_add", "gfix_batch_add_device", "gfix_batch_run",
           "gfix_batch_result", "gfix_batch_destroy", "gfix_coulomb_slices",
           "gfix_coulomb_slices_finish", "gfix_fft_tuning", "gfix_fft_plan",
           "gfix_link_diagnostics", "gfix_gf_check", "gfix_nersc_decode",
           "gfix_nersc_encode",
           "gfix_nersc_error", "gfix_scidac_checksum", "gfix_cut_veclist",
           "gfix_cuts_measure", "gfix_cuts_measure_device", "gfix_cuts_write",
           "gfix_profile_cuts", "gfix_cuts_error", "gfix_cuts_release",
           "gfix_heatbath", "gfix_heatbath_device", "gfix_overrelax",
           "gfix_philox4x32_10", "gfix_update_error", "gfix_update_release",
           "gfix_noalloc_error",
           "gfix_last_error", "gfix_release", "gfix_kernel_launches")

_lib = None


class GfixError(RuntimeError):
    pass


def load(path: Path | str | None = None):
    """Load the library once; raises GfixError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    # GLU_GFIX_LIB selects another build of the same library (e.g. a
    # variant under comparison); the default is the in-tree build
    env = os.environ.get("GLU_GFIX_LIB")
    p = Path(path) if path else (Path(env) if env else LIB)
    if not p.exists():
        raise GfixError(f"{p} is not built: run `python -m glu_b200.build`")
    lib = C.CDLL(str(p))
    for fn in ("gfix_landau", "gfix_landau_device"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                     C.POINTER(GfixResult)]
    for fn in ("gfix_coulomb", "gfix_coulomb_device"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                     C.POINTER(GfixResult), _dp, _szp]
    lib.gfix_landau_sequence.restype = C.c_int
    lib.gfix_landau_sequence.argtypes = [C.POINTER(C.c_void_p), C.c_size_t, _szp,
                                         C.POINTER(GfixParams), C.POINTER(GfixResult)]
    lib.gfix_landau_driver.restype = C.c_int
    lib.gfix_landau_driver.argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                       C.POINTER(GfixResult), _dp, _dp]
    lib.gfix_coulomb_driver.restype = C.c_int
    lib.gfix_coulomb_driver.argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                        C.POINTER(GfixResult), _dp, _dp, _dp, _dp]
    lib.gfix_observables.restype = C.c_int
    lib.gfix_observables.argtypes = [C.c_void_p, _szp, _dp]
    for fn in ("gfix_nersc_decode", "gfix_nersc_encode"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, _szp, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.POINTER(C.c_uint32)]
    lib.gfix_scidac_checksum.restype = C.c_int
    lib.gfix_scidac_checksum.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t,
                                         C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    _ci = C.POINTER(GfixCutInfo)
    lib.gfix_cut_veclist.restype = C.c_long
    lib.gfix_cut_veclist.argtypes = [_szp, _ci, C.POINTER(C.c_int32), C.c_size_t]
    for fn in ("gfix_cuts_measure", "gfix_cuts_measure_device"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, _szp, _ci, C.c_size_t, _dp, _dp, _dp]
    lib.gfix_cuts_write.restype = C.c_int
    lib.gfix_cuts_write.argtypes = [C.c_void_p, _szp, _ci, C.c_char_p, C.c_size_t,
                                    _dp, C.c_char_p, C.c_size_t]
    lib.gfix_profile_cuts.restype = C.c_int
    lib.gfix_profile_cuts.argtypes = [C.c_void_p, _szp, _ci, C.c_int,
                                      C.POINTER(C.c_float)]
    for fn in ("gfix_heatbath", "gfix_heatbath_device"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, _szp, C.c_double, C.c_size_t,
                                     C.c_size_t, C.c_uint64, C.c_uint64, _dp]
    lib.gfix_overrelax.restype = C.c_int
    lib.gfix_overrelax.argtypes = [C.c_void_p, _szp, C.c_size_t]
    _u32p = C.POINTER(C.c_uint32)
    lib.gfix_philox4x32_10.restype = None
    lib.gfix_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
    lib.gfix_update_error.restype = C.c_char_p
    lib.gfix_update_error.argtypes = []
    lib.gfix_update_release.restype = None
    lib.gfix_cuts_error.restype = C.c_char_p
    lib.gfix_cuts_error.argtypes = []
    lib.gfix_cuts_release.restype = None
    lib.gfix_nersc_error.restype = C.c_char_p
    lib.gfix_nersc_error.argtypes = []
    lib.gfix_gf_check.restype = C.c_int
    lib.gfix_gf_check.argtypes = [C.c_void_p, _szp, _dp]
    lib.gfix_link_diagnostics.restype = C.c_int
    lib.gfix_link_diagnostics.argtypes = [C.c_void_p, _szp, _dp]
    lib.gfix_reunit.restype = C.c_int
    lib.gfix_reunit.argtypes = [C.c_void_p, _szp]
    lib.gfix_fourier_accelerate.restype = C.c_int
    lib.gfix_fourier_accelerate.argtypes = [C.c_void_p, _szp, C.c_int]
    lib.gfix_coulomb_slices.restype = C.c_int
    lib.gfix_coulomb_slices.argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                        C.POINTER(GfixResult), _dp, _szp, C.c_void_p,
                                        C.c_void_p]
    lib.gfix_coulomb_slices_finish.restype = C.c_int
    lib.gfix_coulomb_slices_finish.argtypes = [C.c_void_p, _szp, C.c_void_p,
                                               C.c_void_p]
    lib.gfix_fft_tuning.restype = None
    lib.gfix_fft_tuning.argtypes = [C.c_int]
    lib.gfix_fft_plan.restype = C.c_int
    lib.gfix_fft_plan.argtypes = [_szp, C.c_int, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_float)]
    lib.gfix_batch_create.restype = C.c_void_p
    lib.gfix_batch_create.argtypes = [C.POINTER(GfixParams)]
    for fn in ("gfix_batch_add", "gfix_batch_add_device"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [C.c_void_p, C.c_void_p, _szp]
    lib.gfix_batch_run.restype = C.c_int
    lib.gfix_batch_run.argtypes = [C.c_void_p]
    lib.gfix_batch_result.restype = C.c_int
    lib.gfix_batch_result.argtypes = [C.c_void_p, C.c_int, C.POINTER(GfixResult)]
    lib.gfix_batch_destroy.restype = None
    lib.gfix_batch_destroy.argtypes = [C.c_void_p]
    lib.gfix_profile_coulomb.restype = C.c_int
    lib.gfix_profile_coulomb.argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                         C.c_int, _dp, _dp]
    lib.gfix_profile_landau.restype = C.c_int
    lib.gfix_profile_landau.argtypes = [C.c_void_p, _szp, C.POINTER(GfixParams),
                                        C.c_int, _dp, _dp]
    lib.gfix_theta_functional_noalloc.restype = C.c_int
    lib.gfix_theta_functional_noalloc.argtypes = [C.c_void_p, _szp, C.c_void_p,
                                                   C.c_void_p]
    lib.gfix_noalloc_error.restype = C.c_char_p
    lib.gfix_noalloc_error.argtypes = []
    lib.gfix_last_error.restype = C.c_char_p
    lib.gfix_last_error.argtypes = []
    lib.gfix_release.restype = None
    lib.gfix_kernel_launches.restype = C.c_ulonglong
    _lib = lib
    return lib


def check(rc: int):
    if rc != 0:
        msg = _lib.gfix_last_error().decode() if _lib else "library not loaded"
        raise GfixError(msg)
