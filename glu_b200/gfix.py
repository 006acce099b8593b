"""Python mirror of GLU's gauge-fixing interface, backed by libglu_gfix.so.

Names, arguments and return conventions follow the reference:

* ``FACG`` / ``FASD`` -- src/Gfix/FACG.c:341 / :395: return the iteration
  count (``SENTINEL`` = 123456789 on non-convergence) and theta.
* ``Landau`` -- src/Gfix/Landau.c:261: FA solve, reunitarisation.
* ``Coulomb_FA`` / ``Coulomb`` -- src/Gfix/CFACG.c:531 / Coulomb.c:32.
* ``theta_test_lin``, ``gauge_functional`` (src/Gfix/gftests.c:214, :132),
  ``av_plaquette`` (src/Field/plaqs_links.c:243), ``latt_reunitU``
  (src/Geometry/random_config.c:43).

Links are numpy complex128 arrays of shape (V, 4, 3, 3) in GLU's memory
order (site index x fastest), or (Lt, Lz, Ly, Lx, 4, 3, 3); ``dims`` is
(Lx, Ly, Lz, Lt) as in GLU's ``Latt.dims``.  The functions return new
arrays and leave their input untouched.  Every call runs on the GPU; there
is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import GfixParams, GfixResult, check

SENTINEL = 123456789
GLU_FAILURE = (1 << 64) - 1  # GLU_FAILURE (-1) returned through size_t


@dataclass
class FixResult:
    links: np.ndarray
    iters: int
    theta: float
    iters_fp32: int = 0
    gpu_ms: float = 0.0
    traj_theta: np.ndarray = field(default_factory=lambda: np.zeros(0))
    traj_func: np.ndarray = field(default_factory=lambda: np.zeros(0))
    slice_theta: np.ndarray | None = None
    slice_iters: np.ndarray | None = None
    restarts: int = 0


def _dims(dims):
    d = tuple(int(x) for x in dims)
    if len(d) != 4:
        raise ValueError("dims must be (Lx, Ly, Lz, Lt)")
    return (C.c_size_t * 4)(*d), d


def _links(links, d):
    a = np.ascontiguousarray(links, dtype=np.complex128).reshape(-1, 4, 3, 3)
    if a.shape[0] != int(np.prod(d)):
        raise ValueError(f"links hold {a.shape[0]} sites, dims {d} need "
                         f"{int(np.prod(d))}")
    return a.copy()


def _params(alpha, acc, max_iters, algo, sd_fixed, precision, switch, cap,
            max_restarts=0, restart_seed=0, luxury_copies=0, luxury_best=False):
    tt = np.zeros(max(cap, 1))
    tf = np.zeros(max(cap, 1))
    p = GfixParams()
    p.gf_alpha = float(alpha)
    p.accuracy = float(acc)
    p.max_iters = int(max_iters)
    p.algo = {"CG": 0, "FACG": 0, "SD": 1, "FASD": 1}[algo]
    p.sd_fixed_step = int(bool(sd_fixed))
    p.precision = {"FP64": 0, "MIXED": 1}[precision]
    p.switch_theta = float(switch)
    p.traj_theta = tt.ctypes.data_as(C.POINTER(C.c_double)) if cap else None
    p.traj_func = tf.ctypes.data_as(C.POINTER(C.c_double)) if cap else None
    p.traj_cap = int(cap)
    if int(max_restarts) < 0:
        raise ValueError("max_restarts must be >= 0")
    p.max_restarts = int(max_restarts)
    p.restart_seed = int(restart_seed) & 0xFFFFFFFFFFFFFFFF
    if int(luxury_copies) < 0:
        raise ValueError("luxury_copies must be >= 0")
    p.luxury_copies = int(luxury_copies)
    p.luxury_best = int(bool(luxury_best))
    return p, tt, tf


def landau_fix(links, dims, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
               algo="FACG", sd_fixed_step=False, precision="FP64",
               switch_theta=1e-9, traj_cap=0, max_restarts=0,
               restart_seed=0, luxury_copies=0, luxury_best=False) -> FixResult:
    """Landau FA gauge fixing (GLU's FACG/FASD) of a copy of `links`.
    max_restarts > 0 adds GLU's random restarts after a failed solve (its
    Landau driver, src/Gfix/Landau.c:303-340); iters then follows GLU's
    sums and is GLU_FAILURE when every attempt failed.  luxury_copies > 0
    makes each attempt GLU's luxury_copy_fast (Landau.c:92-211): that many
    random gauge copies fixed to 1e-6, the one of largest functional kept
    (smallest with luxury_best, GLU's BEST_COPY) and fixed to accuracy."""
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    p, tt, tf = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                        precision, switch_theta, traj_cap, max_restarts,
                        restart_seed, luxury_copies, luxury_best)
    r = GfixResult()
    check(lib.gfix_landau(U.ctypes.data, cd, C.byref(p), C.byref(r)))
    n = r.traj_len
    return FixResult(U, int(r.iters), float(r.theta), int(r.iters_fp32),
                     float(r.gpu_ms), tt[:n].copy(), tf[:n].copy(),
                     restarts=int(r.restarts))


def landau_sequence(configs, dims, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
                    algo="FACG", sd_fixed_step=False, precision="FP64",
                    switch_theta=1e-9, max_restarts=0, restart_seed=0) -> list:
    """Copies of `configs` (same shape) fixed one after another through
    gfix_landau_sequence, each exactly as landau_fix would fix it; the host
    copies of neighbouring configurations overlap the solves."""
    lib = _lib.load()
    cd, d = _dims(dims)
    Us = [_links(u, d) for u in configs]
    p, _, _ = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                      precision, switch_theta, 0, max_restarts, restart_seed, 0, False)
    n = len(Us)
    ptrs = (C.c_void_p * max(n, 1))(*[u.ctypes.data for u in Us])
    rs = (GfixResult * max(n, 1))()
    check(lib.gfix_landau_sequence(ptrs, n, cd, C.byref(p), rs))
    return [FixResult(U, int(r.iters), float(r.theta), int(r.iters_fp32),
                      float(r.gpu_ms), np.zeros(0), np.zeros(0), restarts=int(r.restarts))
            for U, r in zip(Us, rs)]


def coulomb_fix(links, dims, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
                algo="FACG", sd_fixed_step=False, precision="FP64",
                switch_theta=1e-9, traj_cap=0) -> FixResult:
    """Coulomb FA gauge fixing of all slices (GLU's Coulomb_FA) of a copy of
    `links`.  traj_theta is slice-major: traj_cap // Lt entries per slice,
    NaN past the slice's last FFT round."""
    cd, d = _dims(dims)
    U = _links(links, d)
    r = _coulomb(U.ctypes.data, cd, d, gf_alpha, accuracy, max_iters, algo,
                 sd_fixed_step, precision, switch_theta, traj_cap, False)
    r.links = U
    return r


def coulomb_fix_device(d_links, dims, gf_alpha=0.08, accuracy=1e-14,
                       max_iters=1000, algo="FACG", sd_fixed_step=False,
                       precision="FP64", switch_theta=1e-9,
                       traj_cap=0) -> FixResult:
    """As coulomb_fix on links already in HBM: `d_links` is a device pointer
    (e.g. ``tensor.data_ptr()``) to double[V][4][9][2], fixed in place."""
    cd, d = _dims(dims)
    return _coulomb(int(d_links), cd, d, gf_alpha, accuracy, max_iters, algo,
                    sd_fixed_step, precision, switch_theta, traj_cap, True)


def _coulomb(ptr, cd, d, gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
             precision, switch_theta, traj_cap, device) -> FixResult:
    lib = _lib.load()
    p, tt, tf = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                        precision, switch_theta, traj_cap)
    r = GfixResult()
    sth = np.zeros(d[3])
    sit = np.zeros(d[3], dtype=np.uintp)
    fn = lib.gfix_coulomb_device if device else lib.gfix_coulomb
    check(fn(ptr, cd, C.byref(p), C.byref(r),
             sth.ctypes.data_as(C.POINTER(C.c_double)),
             sit.ctypes.data_as(C.POINTER(C.c_size_t))))
    n = r.traj_len
    return FixResult(None, int(r.iters), float(r.theta), int(r.iters_fp32),
                     float(r.gpu_ms), tt[:n].copy(), tf[:n].copy(), sth,
                     sit.astype(np.int64), int(r.restarts))


def landau_batch(configs, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
                 algo="FACG", sd_fixed_step=False, precision="FP64",
                 switch_theta=1e-9) -> list:
    """Landau FA gauge fixing of many configurations in one batch
    (gfix_batch_*): `configs` is a sequence of (links, dims); returns one
    FixResult per configuration, in order, each equal to landau_fix's."""
    lib = _lib.load()
    p, _, _ = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                      precision, switch_theta, 0)
    b = lib.gfix_batch_create(C.byref(p))
    if not b:
        check(-1)
    try:
        bufs = []
        for links, dims in configs:
            cd, d = _dims(dims)
            U = _links(links, d)
            bufs.append((U, cd))
            if lib.gfix_batch_add(b, U.ctypes.data, cd) < 0:
                check(-1)
        check(lib.gfix_batch_run(b))
        out = []
        for i, (U, _) in enumerate(bufs):
            r = GfixResult()
            check(lib.gfix_batch_result(b, i, C.byref(r)))
            out.append(FixResult(U, int(r.iters), float(r.theta),
                                 int(r.iters_fp32), float(r.gpu_ms),
                                 restarts=int(r.restarts)))
        return out
    finally:
        lib.gfix_batch_destroy(b)


# --- GLU-named entry points -------------------------------------------------

def FACG(links, dims, gf_alpha, acc, max_iters, **kw):
    """src/Gfix/FACG.c:341 -> (links, iters, theta)."""
    r = landau_fix(links, dims, gf_alpha, acc, max_iters, "FACG", **kw)
    return r.links, r.iters, r.theta


def FASD(links, dims, gf_alpha, acc, max_iters, **kw):
    """src/Gfix/FACG.c:395 -> (links, iters, theta)."""
    r = landau_fix(links, dims, gf_alpha, acc, max_iters, "FASD", **kw)
    return r.links, r.iters, r.theta


GF_GLU_FAILURES = 7  # src/Headers/GLU_definitions.h:400-402


@dataclass
class DriverResult:
    links: np.ndarray
    iters: int
    theta: float
    restarts: int
    plaquette: float = 0.0
    functional: float = 0.0
    theta_test: float = 0.0
    diagnostics: dict = field(default_factory=dict)


def landau_driver(links, dims, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
                  algo="FACG", sd_fixed_step=False, precision="FP64",
                  switch_theta=1e-9, max_restarts=GF_GLU_FAILURES - 1,
                  restart_seed=1, luxury_copies=0, luxury_best=False) -> DriverResult:
    """GLU's Landau driver (src/Gfix/Landau.c:261-374) in one pass on the GPU
    (gfix_landau_driver): the solve with random restarts, then the
    reunitarised links and output_fixing_info's numbers."""
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    p, _, _ = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                      precision, switch_theta, 0, max_restarts, restart_seed,
                      luxury_copies, luxury_best)
    r = GfixResult()
    obs = np.zeros(3)
    dg = np.zeros(6)
    check(lib.gfix_landau_driver(U.ctypes.data, cd, C.byref(p), C.byref(r),
                                 obs.ctypes.data_as(C.POINTER(C.c_double)),
                                 dg.ctypes.data_as(C.POINTER(C.c_double))))
    return DriverResult(U, int(r.iters), float(r.theta), int(r.restarts),
                        float(obs[2]), float(obs[1]), float(obs[0]),
                        dict(splink=dg[0], tlink=dg[1], link=dg[2], link_max=dg[3],
                             const_lin=dg[4], const_log=dg[5]))


def coulomb_driver(links, dims, gf_alpha=0.08, accuracy=1e-14, max_iters=1000,
                   algo="FACG", sd_fixed_step=False, precision="FP64",
                   switch_theta=1e-9):
    """GLU's Coulomb driver (src/Gfix/Coulomb.c:32-106) in one pass on the
    GPU (gfix_coulomb_driver): (initial, final) DriverResult pair, the final
    one holding the fixed, reunitarised links."""
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    p, _, _ = _params(gf_alpha, accuracy, max_iters, algo, sd_fixed_step,
                      precision, switch_theta, 0)
    r = GfixResult()
    o0, d0, o1, d1 = np.zeros(3), np.zeros(6), np.zeros(3), np.zeros(6)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    check(lib.gfix_coulomb_driver(U.ctypes.data, cd, C.byref(p), C.byref(r),
                                  dp(o0), dp(d0), dp(o1), dp(d1)))
    diag = lambda g: dict(splink=g[0], tlink=g[1], link=g[2], link_max=g[3],  # noqa: E731
                          const_lin=g[4], const_log=g[5])
    first = DriverResult(None, 0, 0.0, 0, float(o0[2]), float(o0[1]), float(o0[0]),
                         diag(d0))
    last = DriverResult(U, int(r.iters), float(r.theta), int(r.restarts),
                        float(o1[2]), float(o1[1]), float(o1[0]), diag(d1))
    return first, last


def Landau(links, dims, gf_alpha, accuracy, max_iters, **kw):
    """src/Gfix/Landau.c:261 -> (links, iters): the solve with GLU's random
    restarts and the final reunitarisation; iters = GLU_FAILURE when every
    attempt failed."""
    r = landau_driver(links, dims, gf_alpha, accuracy, max_iters, **kw)
    return r.links, r.iters


def Coulomb_FA(links, dims, gf_alpha, accuracy, max_iters, facg=True, **kw):
    """src/Gfix/CFACG.c:531 -> (links, iters)."""
    r = coulomb_fix(links, dims, gf_alpha, accuracy, max_iters,
                    "FACG" if facg else "FASD", **kw)
    return r.links, r.iters


def Coulomb(links, dims, gf_alpha, accuracy, max_iters, **kw):
    """src/Gfix/Coulomb.c:32 -> (links, iters), links reunitarised."""
    _, r = coulomb_driver(links, dims, gf_alpha, accuracy, max_iters, **kw)
    return r.links, r.iters


def observables(links, dims):
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    out = np.zeros(3)
    check(lib.gfix_observables(U.ctypes.data, cd,
                               out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def theta_test_lin(links, dims):
    return float(observables(links, dims)[0])


def gauge_functional(links, dims):
    return float(observables(links, dims)[1])


def av_plaquette(links, dims):
    return float(observables(links, dims)[2])


def latt_reunitU(links, dims):
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    check(lib.gfix_reunit(U.ctypes.data, cd))
    return U


def fourier_accelerate(fields, dims, ndim=4):
    """The GPU FOURIER_ACCELERATE3 (ndim 4, fields of shape (4, V)) or
    FOURIER_ACCELERATE2 (ndim 3, one time slice, shape (4, Lx Ly Lz))."""
    lib = _lib.load()
    cd, d = _dims(dims)
    f = np.ascontiguousarray(fields, dtype=np.complex128).copy()
    check(lib.gfix_fourier_accelerate(f.ctypes.data, cd, ndim))
    return f


def link_diagnostics(links, dims) -> dict:
    """GLU's post-fix link diagnostics (gfix_link_diagnostics): spatial and
    temporal average link trace (all_links), average and largest link trace
    (indivlinks, both / NC) and the linear and logarithmic temporal
    constancy (const_time)."""
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    out = np.zeros(6)
    check(lib.gfix_link_diagnostics(U.ctypes.data, cd,
                                    out.ctypes.data_as(C.POINTER(C.c_double))))
    return dict(splink=out[0], tlink=out[1], link=out[2], link_max=out[3],
                const_lin=out[4], const_log=out[5])


def gf_check(links, dims) -> dict:
    """GLU's gauge-fixing accuracy report (gf_check, OBS_wrap.c:93-126):
    theta_test_lin / theta_test_log and their largest local values over the
    four (landau_*) and the three spatial (coulomb_*) directions, and the
    temporal constancy of both definitions."""
    lib = _lib.load()
    cd, d = _dims(dims)
    U = _links(links, d)
    o = np.zeros(10)
    check(lib.gfix_gf_check(U.ctypes.data, cd, o.ctypes.data_as(C.POINTER(C.c_double))))
    return dict(landau_lin=o[0], landau_lin_max=o[1], landau_log=o[2],
                landau_log_max=o[3], const_lin=o[4], const_log=o[5],
                coulomb_lin=o[6], coulomb_lin_max=o[7], coulomb_log=o[8],
                coulomb_log_max=o[9])


def gf_check_report(r: dict) -> str:
    """The [GFACC] lines GLU prints for gf_check's numbers."""
    return ("[GFACC] Looking at Landau Gauge-Fixing Information \n"
            f"[GFACC LANDAU]      LIN :: {r['landau_lin']:1.6e} \n"
            f"[GFACC MAX LANDAU]  LIN :: {r['landau_lin_max']:1.6e} \n"
            f"[GFACC LANDAU]      LOG :: {r['landau_log']:1.6e} \n"
            f"[GFACC MAX LANDAU]  LOG :: {r['landau_log_max']:1.6e} \n"
            f"[GFACC] Temporal constance || LIN {r['const_lin']:e} || Log {r['const_log']:e} "
            "\n[GFACC] Looking at Coulomb Gauge-Fixing Information \n"
            f"[GFACC COULOMB]     LIN :: {r['coulomb_lin']:1.6e} \n"
            f"[GFACC MAX COULOMB] LIN :: {r['coulomb_lin_max']:1.6e} \n"
            f"[GFACC COULOMB]     LOG :: {r['coulomb_log']:1.6e} \n"
            f"[GFACC MAX COULOMB] LOG :: {r['coulomb_log_max']:1.6e} \n\n")


def fft_tuning(on: bool):
    """Autotuned FFT plans per lattice shape (True) or the fixed default
    plans (False, bit-reproducible); see gfix_fft_tuning."""
    _lib.load().gfix_fft_tuning(1 if on else 0)


def fft_plan(dims, coulomb=False, precision="FP64"):
    """((xy pass, zt tile width, zt pass), (xy ms, zt ms)) of a shape's
    workspace: pass -1 = compile-time, else the generic pass's radix order;
    times 0 unless tuned."""
    lib = _lib.load()
    cd, _ = _dims(dims)
    plan = (C.c_int * 3)()
    ms = (C.c_float * 2)()
    check(lib.gfix_fft_plan(cd, int(bool(coulomb)), {"FP64": 0, "MIXED": 1}[precision],
                            plan, ms))
    return tuple(plan), tuple(ms)


def kernel_launches() -> int:
    return int(_lib.load().gfix_kernel_launches())


def release():
    _lib.load().gfix_release()
