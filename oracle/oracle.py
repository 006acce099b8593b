"""ctypes access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Two libraries are wrapped:

* ``Oracle``  -- ``oracle/_build/liboracle.so``, our C restatement of GLU's
  Fourier-accelerated Landau/Coulomb gauge fixing (gfix_oracle.c).
* ``Reference`` -- ``oracle/_ref/libglu_ref.so`` (and ``libglu_ref_sd.so``
  for a GLU_GFIX_SD build), the reference GLU compiled from its own sources
  by ``oracle/Makefile`` plus the ctypes harness ``ref_harness.c``.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker or the timed CPU
baseline.  The product package ``glu_b200`` never does.

Links are numpy complex128 arrays of shape (V, 4, 3, 3) in GLU's memory
order (site index with x fastest); dims are (Lx, Ly, Lz, Lt).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libglu_ref.so"
REF_SD_SO = HERE / "_ref" / "libglu_ref_sd.so"
REF_BIN = HERE / "_ref" / "glu"

SENTINEL = 123456789

_dp = C.POINTER(C.c_double)
_sz = C.c_size_t
_szp = C.POINTER(C.c_size_t)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _dims(dims):
    return (C.c_size_t * 4)(*[int(d) for d in dims])


def _links_buf(links: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(links, dtype=np.complex128)
    return a.reshape(-1, 4, 3, 3)


class Oracle:
    """Our C restatement (oracle/gfix_oracle.c)."""

    def __init__(self, path: Path | str = ORACLE_SO):
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.orc_landau_fa.restype = _sz
        L.orc_landau_fa.argtypes = [_dp, _szp, C.c_double, C.c_double, _sz,
                                    C.c_int, C.c_int, _dp, _dp, _dp, _sz, _szp]
        L.orc_coulomb_fa.restype = _sz
        L.orc_coulomb_fa.argtypes = [_dp, _szp, C.c_double, C.c_double, _sz,
                                     C.c_int, C.c_int, _dp, _szp, _dp, _sz,
                                     _szp, _szp]
        for n in ("orc_theta_test_lin", "orc_gauge_functional", "orc_plaquette"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [_dp, _szp]
        L.orc_reunit_links.argtypes = [_dp, _sz]
        L.orc_derivative.restype = C.c_double
        L.orc_derivative.argtypes = [_dp, _szp, _dp]
        L.orc_fourier_accelerate.argtypes = [_dp, _szp, C.c_int]
        L.orc_psq.argtypes = [_dp, _szp, C.c_int]
        L.orc_dft.argtypes = [_dp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.orc_sum_pr.argtypes = [_dp, _dp, _sz, _dp]
        L.orc_line_search_probes.restype = C.c_double
        L.orc_line_search_probes.argtypes = [_dp, _szp, _dp, _dp]
        L.orc_link_update.argtypes = [_dp, _szp, _dp, C.c_double]
        L.orc_gauge_matrix.argtypes = [_dp, _sz, _sz, C.c_double, _dp]
        L.orc_gram_reunit.argtypes = [_dp]
        L.orc_approx_minimum.restype = C.c_double
        L.orc_approx_minimum.argtypes = [_dp, _dp]

    # --- solvers ---------------------------------------------------------
    def landau(self, links, dims, alpha, acc, max_iters, algo="FACG",
               sd_fixed_step=False, traj_cap=0):
        U = _links_buf(links).copy()
        th = np.zeros(1)
        tt = np.zeros(max(traj_cap, 1))
        tf = np.zeros(max(traj_cap, 1))
        n = _sz(0)
        it = self.lib.orc_landau_fa(
            _ptr(U), _dims(dims), alpha, acc, max_iters,
            0 if algo == "FACG" else 1, int(sd_fixed_step), _ptr(th),
            _ptr(tt) if traj_cap else None, _ptr(tf) if traj_cap else None,
            traj_cap, C.byref(n))
        return dict(links=U, iters=int(it), theta=float(th[0]),
                    traj_theta=tt[: n.value].copy(), traj_func=tf[: n.value].copy())

    def coulomb(self, links, dims, alpha, acc, max_iters, algo="FACG",
                sd_fixed_step=False, traj_cap=0):
        U = _links_buf(links).copy()
        T = int(dims[3])
        sth = np.zeros(T)
        sit = np.zeros(T, dtype=np.uintp)
        tt = np.zeros(max(traj_cap, 1))
        n = _sz(0)
        rs = _sz(0)
        it = self.lib.orc_coulomb_fa(
            _ptr(U), _dims(dims), alpha, acc, max_iters,
            1 if algo == "FACG" else 0, int(sd_fixed_step), _ptr(sth),
            sit.ctypes.data_as(_szp), _ptr(tt) if traj_cap else None,
            traj_cap, C.byref(n), C.byref(rs))
        return dict(links=U, iters=int(it), slice_theta=sth,
                    slice_iters=sit.astype(np.int64),
                    traj_theta=tt[: n.value].copy(), restarts=int(rs.value))

    # --- pieces ------------------------------------------------------------
    def theta_test_lin(self, links, dims):
        return self.lib.orc_theta_test_lin(_ptr(_links_buf(links)), _dims(dims))

    def gauge_functional(self, links, dims):
        return self.lib.orc_gauge_functional(_ptr(_links_buf(links)), _dims(dims))

    def plaquette(self, links, dims):
        return self.lib.orc_plaquette(_ptr(_links_buf(links)), _dims(dims))

    def reunit(self, links):
        U = _links_buf(links).copy()
        self.lib.orc_reunit_links(_ptr(U), U.shape[0] * 4)
        return U

    def derivative(self, links, dims):
        V = int(np.prod(dims))
        f = np.zeros((4, V), dtype=np.complex128)
        th = self.lib.orc_derivative(_ptr(_links_buf(links)), _dims(dims), _ptr(f))
        return f, th

    def fourier_accelerate(self, fields, dims, ndim=4):
        f = np.ascontiguousarray(fields, dtype=np.complex128).copy()
        self.lib.orc_fourier_accelerate(_ptr(f), _dims(dims), ndim)
        return f

    def psq(self, dims, ndim=4):
        vol = int(np.prod(dims[:ndim]))
        p = np.zeros(vol)
        self.lib.orc_psq(_ptr(p), _dims(dims), ndim)
        return p

    def dft(self, data, sign):
        a = np.ascontiguousarray(data, dtype=np.complex128).copy()
        n = (C.c_int * a.ndim)(*a.shape)
        self.lib.orc_dft(_ptr(a), a.ndim, n, sign)
        return a

    def sum_pr(self, fin, fold):
        fin = np.ascontiguousarray(fin, dtype=np.complex128)
        fold = np.ascontiguousarray(fold, dtype=np.complex128)
        out = np.zeros(2)
        self.lib.orc_sum_pr(_ptr(fin), _ptr(fold), fin.shape[1], _ptr(out))
        return out

    def line_search(self, links, dims, sn):
        val = np.zeros(3)
        sn = np.ascontiguousarray(sn, dtype=np.complex128)
        a = self.lib.orc_line_search_probes(_ptr(_links_buf(links)), _dims(dims),
                                            _ptr(sn), _ptr(val))
        return a, val

    def link_update(self, links, dims, sn, alpha):
        U = _links_buf(links).copy()
        sn = np.ascontiguousarray(sn, dtype=np.complex128)
        self.lib.orc_link_update(_ptr(U), _dims(dims), _ptr(sn), alpha)
        return U

    def gauge_matrix(self, fields, i, alpha):
        f = np.ascontiguousarray(fields, dtype=np.complex128)
        g = np.zeros(9, dtype=np.complex128)
        self.lib.orc_gauge_matrix(_ptr(f), f.shape[1], i, alpha, _ptr(g))
        return g.reshape(3, 3)

    def approx_minimum(self, alphas, vals):
        a = np.ascontiguousarray(alphas, dtype=np.float64)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        return self.lib.orc_approx_minimum(_ptr(a), _ptr(v))


class Reference:
    """GLU itself, compiled from its sources (oracle/Makefile)."""

    def __init__(self, sd_build: bool = False, path: Path | str | None = None):
        p = path or (REF_SD_SO if sd_build else REF_SO)
        # GLU keeps its state in globals: one library file is one lattice,
        # so instances of the same build share it
        self.lib = C.CDLL(str(p), mode=os.RTLD_LOCAL)
        L = self.lib
        L.ref_setup.restype = C.c_int
        L.ref_setup.argtypes = [_szp, C.c_int, C.c_double, C.c_uint]
        L.ref_read_file.restype = C.c_int
        L.ref_read_file.argtypes = [C.c_char_p, _szp, C.c_int]
        L.ref_set_alpha.argtypes = [C.c_double]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_volume.restype = _sz
        L.ref_put_links.argtypes = [_dp]
        L.ref_get_links.argtypes = [_dp]
        for n in ("ref_theta_test_lin", "ref_gauge_functional",
                  "ref_av_plaquette", "ref_fft_seconds"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = []
        L.ref_read_file_as.restype = C.c_int
        L.ref_read_file_as.argtypes = [C.c_char_p, _szp, C.c_int, C.c_int]
        L.ref_write_config.restype = C.c_int
        L.ref_write_config.argtypes = [C.c_char_p, C.c_int, C.c_char_p]
        L.ref_output_code.restype = C.c_int
        L.ref_output_code.argtypes = [C.c_char_p]
        L.ref_all_links.restype = C.c_double
        L.ref_all_links.argtypes = [_dp, _dp]
        L.ref_indivlinks.restype = C.c_double
        L.ref_indivlinks.argtypes = [_dp]
        L.ref_const_time.restype = None
        L.ref_const_time.argtypes = [_dp, _dp]
        L.ref_gf_check.restype = None
        L.ref_gf_check.argtypes = [_dp]
        L.ref_landau_fa.restype = _sz
        L.ref_landau_fa.argtypes = [C.c_int, C.c_double, _sz, _dp, _dp, _dp,
                                    _sz, _szp]
        L.ref_coulomb_fa.restype = _sz
        L.ref_coulomb_fa.argtypes = [C.c_int, C.c_double, _sz, _dp, _sz, _szp]
        L.ref_landau.restype = _sz
        L.ref_landau.argtypes = [C.c_double, _sz, C.c_char_p]
        L.ref_coulomb.restype = _sz
        L.ref_coulomb.argtypes = [C.c_double, _sz]
        L.ref_veclist.restype = C.c_long
        L.ref_veclist.argtypes = [C.c_int, C.c_int, _sz, _sz, C.c_double,
                                  C.POINTER(C.c_int), _szp, _sz]
        L.ref_cut_output_name.restype = C.c_int
        L.ref_cut_output_name.argtypes = [C.c_int, C.c_int, _sz, C.c_int, _sz,
                                          C.c_double, _sz, C.c_char_p, _sz]
        L.ref_overrelax.restype = C.c_int
        L.ref_overrelax.argtypes = [_sz]
        L.ref_heatbath.restype = C.c_int
        L.ref_heatbath.argtypes = [C.c_double, _sz, _sz, _dp]
        L.ref_cuts.restype = C.c_int
        L.ref_cuts.argtypes = [C.c_int, C.c_int, _sz, C.c_int, _sz, C.c_double,
                               _sz, C.c_char_p]
        self.dims = None

    def setup(self, dims, nthreads=1, alpha=0.08, seed=1):
        self.dims = tuple(int(d) for d in dims)
        if self.lib.ref_setup(_dims(dims), nthreads, alpha, seed) != 0:
            raise RuntimeError("reference lattice allocation failed")

    def read_file(self, path, nthreads=1, ildg=False):
        d = (C.c_size_t * 4)()
        if self.lib.ref_read_file_as(str(path).encode(), d, nthreads,
                                     1 if ildg else 0) != 0:
            raise RuntimeError(f"reference could not read {path}")
        self.dims = tuple(d)
        return self.get_links()

    def set_alpha(self, a):
        self.lib.ref_set_alpha(a)

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def put_links(self, links):
        U = _links_buf(links)
        self.lib.ref_put_links(_ptr(U))

    def get_links(self):
        V = int(self.lib.ref_volume())
        U = np.zeros((V, 4, 3, 3), dtype=np.complex128)
        self.lib.ref_get_links(_ptr(U))
        return U

    def theta_test_lin(self):
        return self.lib.ref_theta_test_lin()

    def gauge_functional(self):
        return self.lib.ref_gauge_functional()

    def plaquette(self):
        return self.lib.ref_av_plaquette()

    def write(self, path, storage="ILDG", details="glu_b200 fixture"):
        """GLU's write_configuration of the lattice in place (which
        reunitarises it first)."""
        code = self.lib.ref_output_code(storage.encode())
        if code < 0 or self.lib.ref_write_config(str(path).encode(), code,
                                                 details.encode()) != 0:
            raise RuntimeError(f"reference could not write {path}")

    def diagnostics(self):
        """(splink, tlink, all, indivlinks average, indivlinks max,
        const_time lin, const_time log) of the lattice in place."""
        sp, t, mx, lin, lg = (np.zeros(1) for _ in range(5))
        al = self.lib.ref_all_links(_ptr(sp), _ptr(t))
        avg = self.lib.ref_indivlinks(_ptr(mx))
        self.lib.ref_const_time(_ptr(lin), _ptr(lg))
        return (float(sp[0]), float(t[0]), float(al), float(avg), float(mx[0]),
                float(lin[0]), float(lg[0]))

    def gf_check(self):
        """GLU's gf_check numbers of the lattice in place: (Landau lin, its
        max, Landau log, its max, const_time lin, log, Coulomb lin, max,
        Coulomb log, max)."""
        out = np.zeros(10)
        self.lib.ref_gf_check(_ptr(out))
        return out

    def landau_fa(self, acc, max_iters, algo="FACG", traj_cap=0):
        th = np.zeros(1)
        tt = np.zeros(max(traj_cap, 1))
        tf = np.zeros(max(traj_cap, 1))
        n = _sz(0)
        it = self.lib.ref_landau_fa(0 if algo == "FACG" else 1, acc, max_iters,
                                    _ptr(th), _ptr(tt) if traj_cap else None,
                                    _ptr(tf) if traj_cap else None, traj_cap,
                                    C.byref(n))
        return dict(iters=int(it), theta=float(th[0]),
                    traj_theta=tt[: n.value].copy(),
                    traj_func=tf[: n.value].copy())

    def coulomb_fa(self, acc, max_iters, algo="FACG", traj_cap=0):
        tt = np.zeros(max(traj_cap, 1))
        n = _sz(0)
        it = self.lib.ref_coulomb_fa(1 if algo == "FACG" else 0, acc, max_iters,
                                     _ptr(tt) if traj_cap else None, traj_cap,
                                     C.byref(n))
        return dict(iters=int(it), traj_theta=tt[: n.value].copy())

    def fft_seconds(self):
        return self.lib.ref_fft_seconds()

    # configuration generation (src/Update)
    def overrelax(self, sweeps):
        """GLU's OR_lattice sweeps on the lattice in place."""
        if self.lib.ref_overrelax(sweeps) != 0:
            raise RuntimeError("reference over-relaxation failed")

    def heatbath(self, beta, iterations, n_or=0):
        """GLU's heatbath steps on the lattice in place (its own generator,
        seeded by setup's seed); the plaquette after every step."""
        plaq = np.zeros(max(iterations, 1))
        if self.lib.ref_heatbath(beta, iterations, n_or, _ptr(plaq)) != 0:
            raise RuntimeError("reference heatbath failed")
        return plaq[:iterations]

    # momentum-space cuts (src/Cuts/cuts.c:110-184)
    def veclist(self, dir, type, max_mom, angle=0, cyl_width=1.0):
        """(MOM (n, 4), idx (n,)) of compute_veclist for the current dims."""
        V = int(np.prod(self.dims))
        mom = np.zeros((V, 4), dtype=np.int32)
        idx = np.zeros(V, dtype=np.uint64)
        n = self.lib.ref_veclist(dir, type, max_mom, angle, cyl_width,
                                 mom.ctypes.data_as(C.POINTER(C.c_int)),
                                 idx.ctypes.data_as(_szp), V)
        return mom[:n].astype(np.int64), idx[:n].astype(np.int64)

    def cut_output_name(self, dir, type, max_mom, definition=0, angle=0,
                        cyl_width=1.0, flow=0):
        buf = C.create_string_buffer(1024)
        self.lib.ref_cut_output_name(dir, type, max_mom, definition, angle,
                                     cyl_width, flow, buf, 1024)
        return buf.value.decode()

    def cuts(self, where, dir, type, max_mom, definition=0, angle=0,
             cyl_width=1.0, flow=0):
        """GLU's cuts_struct on the lattice in place; returns the path of
        the file it wrote (the lattice then holds momentum-space fields)."""
        name = self.cut_output_name(dir, type, max_mom, definition, angle,
                                    cyl_width, flow)
        if self.lib.ref_cuts(dir, type, max_mom, definition, angle, cyl_width,
                             flow, str(where).encode()) != 0:
            raise RuntimeError("reference cuts_struct failed")
        return Path(where) / name


def available() -> dict:
    return {"oracle": ORACLE_SO.exists(), "reference": REF_SO.exists(),
            "reference_sd": REF_SD_SO.exists(), "glu": REF_BIN.exists()}
