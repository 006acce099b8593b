"""Quenched SU(3) configuration generation on the GPU: GLU's heatbath +
over-relaxation update (MODE = HEATBATH, hb_update in src/Update/KPHB.c),
through gfix_heatbath / gfix_overrelax.

Links are numpy complex128 arrays (V, 4, 3, 3) in GLU's site order (x
fastest), dims (Lx, Ly, Lz, Lt), all even.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class UpdateError(RuntimeError):
    pass


def _dims(dims):
    return (C.c_size_t * 4)(*[int(d) for d in dims])


def _links(links, dims):
    V = int(np.prod([int(d) for d in dims]))
    U = np.array(links, dtype=np.complex128, copy=True, order="C")
    if U.size != V * 36:
        raise ValueError(f"links hold {U.size // 36} sites, dims {tuple(dims)} need {V}")
    return U.reshape(V, 4, 3, 3)


def unit_config(dims) -> np.ndarray:
    """GLU's UNIT_GAUGE start: every link the identity."""
    V = int(np.prod([int(d) for d in dims]))
    U = np.zeros((V, 4, 3, 3), dtype=np.complex128)
    for k in range(3):
        U[..., k, k] = 1.0
    return U


def heatbath(links, dims, beta, iterations, n_or=4, seed=1, first_iteration=0):
    """`iterations` steps of one heatbath sweep and n_or over-relaxation
    sweeps on a copy of `links` (GLU's update_lattice, KPHB.c:83-99);
    returns (links, plaquette after every step).  A run continued with
    first_iteration = the number of steps done equals the uninterrupted one."""
    lib = _lib.load()
    U = _links(links, dims)
    plaq = np.zeros(max(int(iterations), 1))
    rc = lib.gfix_heatbath(U.ctypes.data, _dims(dims), float(beta), int(iterations),
                           int(n_or), int(seed) & 0xFFFFFFFFFFFFFFFF, int(first_iteration),
                           plaq.ctypes.data_as(_lib._dp))
    if rc != 0:
        raise UpdateError(lib.gfix_update_error().decode())
    return U, plaq[: int(iterations)]


def heatbath_device(links, dims, beta, iterations, n_or=4, seed=1, first_iteration=0):
    """The same in place on links in device memory (a CUDA tensor holding
    GLU's layout); returns the plaquettes."""
    lib = _lib.load()
    plaq = np.zeros(max(int(iterations), 1))
    rc = lib.gfix_heatbath_device(links.data_ptr(), _dims(dims), float(beta), int(iterations),
                                  int(n_or), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                  int(first_iteration), plaq.ctypes.data_as(_lib._dp))
    if rc != 0:
        raise UpdateError(lib.gfix_update_error().decode())
    return plaq[: int(iterations)]


def overrelax(links, dims, sweeps=1):
    """`sweeps` over-relaxation sweeps (GLU's OR_lattice) on a copy."""
    lib = _lib.load()
    U = _links(links, dims)
    if lib.gfix_overrelax(U.ctypes.data, _dims(dims), int(sweeps)) != 0:
        raise UpdateError(lib.gfix_update_error().decode())
    return U


def philox4x32_10(ctr, key):
    """The generator's block function (host): 4 words of counter, 2 of key."""
    lib = _lib.load()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.gfix_philox4x32_10(c, k, o)
    return tuple(int(x) for x in o)
