"""GLU's own entry points, called as GLU calls them: a struct site lattice
(each lat[i].O[mu] a separate 3x3 complex matrix), the dimensions and
GF_TUNE in the global Latt, the FFT fields in a struct fftw_stuff.  These
are the symbols a GLU build links in place of the archive members FACG.o,
Landau.o, Coulomb.o and CFACG.o; the last tests run GLU's own program
relinked that way (oracle/_ref/glu_gpu) beside the stock one
(oracle/_ref/glu) on the same input file and configuration.
"""
import ctypes as C
import os
import re
import subprocess
import time
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import _lib, gfix  # noqa: E402
from glu_structs import (GLU_INPUT as INPUT, FftwStuff, Site, SiteLattice,  # noqa: E402
                         fftw_fields, flush_c_stdio, set_latt)

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
GLU_FAILURE = (1 << 64) - 1
_szt = C.c_size_t
_PS = C.POINTER(Site)
_PF = C.POINTER(FftwStuff)


@pytest.fixture(scope="module")
def lib():
    L = _lib.load()
    L.FACG.restype = _szt
    L.FACG.argtypes = [_PS, _PF, C.POINTER(C.c_double), C.c_double, _szt]
    L.FASD.restype = _szt
    L.FASD.argtypes = [_PS, _PF, C.POINTER(C.c_double), C.c_double, _szt]
    L.Landau.restype = _szt
    L.Landau.argtypes = [_PS, C.c_double, _szt, C.c_char_p]
    L.Coulomb.restype = _szt
    L.Coulomb.argtypes = [_PS, C.c_double, _szt]
    L.Coulomb_FA.restype = _szt
    L.Coulomb_FA.argtypes = [_PS, _PF, C.c_double, _szt, C.c_int]
    L.FOURIER_ACCELERATE3.restype = None
    L.FOURIER_ACCELERATE3.argtypes = [_PF]
    L.FOURIER_ACCELERATE2.restype = None
    L.FOURIER_ACCELERATE2.argtypes = [_PF]
    return L


def _dims(g):
    return tuple(int(d) for d in g["dims"])


@pytest.mark.parametrize("name", ["FACG", "FASD"])
def test_facg_fasd_on_a_site_lattice_equal_the_flat_solve(lib, lat400, name):
    """FACG / FASD (src/Gfix/FACG.c:341-446) on lat[i].O[mu]: the same
    iteration count, theta and links, bit for bit, as gfix_landau on the
    contiguous links; GLU's own iteration count within its reproducibility."""
    d = _dims(lat400)
    set_latt(lib, d, gf_alpha=0.08)
    L = SiteLattice(lat400["links"])
    th = C.c_double(0.0)
    it = getattr(lib, name)(L.sites, None, C.byref(th), 1e-14, 650)
    flat = gfix.landau_fix(lat400["links"], d, 0.08, 1e-14, 650, name)
    assert it == flat.iters
    assert th.value == flat.theta
    assert np.array_equal(L.U, flat.links)
    if name == "FACG":
        assert abs(it - int(lat400["landau_facg_iters"])) <= 3
    assert th.value < 1e-14
    # non-convergence: FACG returns the sentinel, FASD the sentinel plus the
    # run's iterations (src/Gfix/FACG.c:381, 429-437); links written back
    L2 = SiteLattice(lat400["links"])
    bad = gfix.SENTINEL + (3 if name == "FASD" else 0)
    assert getattr(lib, name)(L2.sites, None, C.byref(th), 1e-14, 3) == bad
    assert not np.array_equal(L2.U, lat400["links"])


def test_fourier_accelerate3_on_fftw_stuff(lib, oracle, lat400):
    """FOURIER_ACCELERATE3 (FACG.c:77-95) on the four fields FFTW->in."""
    d = _dims(lat400)
    set_latt(lib, d)
    rng = np.random.default_rng(3)
    V = int(np.prod(d))
    f = rng.normal(size=(4, V)) + 1j * rng.normal(size=(4, V))
    st, keep = fftw_fields(f.copy())  # transformed in place
    lib.FOURIER_ACCELERATE3(C.byref(st))
    ref = oracle.fourier_accelerate(f, d, 4)
    assert np.abs(keep[0] - ref).max() < 1e-13 * np.abs(ref).max()


def test_fourier_accelerate2_on_fftw_stuff(lib, oracle, lat400):
    """FOURIER_ACCELERATE2 (CFACG.c:69-88) on one time slice."""
    d = _dims(lat400)
    set_latt(lib, d)
    rng = np.random.default_rng(4)
    n = d[0] * d[1] * d[2]
    f = rng.normal(size=(4, n)) + 1j * rng.normal(size=(4, n))
    st, keep = fftw_fields(f.copy())  # transformed in place
    lib.FOURIER_ACCELERATE2(C.byref(st))
    ref = oracle.fourier_accelerate(f, d, 3)
    assert np.abs(keep[0] - ref).max() < 1e-13 * np.abs(ref).max()


def test_landau_driver_on_a_site_lattice(lib, lat400, capfd):
    """Landau (src/Gfix/Landau.c:261-374): the fix, the reunitarised links
    and GLU's "[GF]" summary, with GLU's plaquette and iteration count."""
    d = _dims(lat400)
    set_latt(lib, d, gf_alpha=0.08, seed=1)
    L = SiteLattice(lat400["links"])
    it = lib.Landau(L.sites, 1e-14, 650, b"unused")
    flush_c_stdio()
    out = capfd.readouterr().out
    flat = gfix.landau_fix(lat400["links"], d, 0.08, 1e-14, 650, "FACG")
    assert it == flat.iters
    assert np.array_equal(L.U, gfix.latt_reunitU(flat.links, d))
    assert abs(it - int(lat400["landau_facg_iters"])) <= 3
    m = re.search(r"\[GF\] Plaquette :: ([0-9.]+)", out)
    assert m and abs(float(m.group(1)) - lat400["plaquette"]) < 1e-13
    assert f"[GF] Iters :: {it}" in out
    m = re.search(r"\[GF\] Functional :: ([0-9.]+)", out)
    assert m and abs(float(m.group(1)) - gfix.gauge_functional(L.U, d)) < 1e-14


def test_landau_driver_exhausts_its_restarts(lib, lat400, capfd):
    """Every attempt fails (MAX_ITERS 3): GLU_FAILURE after
    GF_GLU_FAILURES - 1 = 6 restarts, each reported as GLU reports it; the
    links are the last attempt's, on the input's gauge orbit."""
    d = _dims(lat400)
    set_latt(lib, d, gf_alpha=0.08, seed=5)
    L = SiteLattice(lat400["links"])
    assert lib.Landau(L.sites, 1e-14, 3, b"unused") == GLU_FAILURE
    flush_c_stdio()
    cap = capfd.readouterr()
    assert cap.err.count("Randomly-restarting") == 7  # attempt 0 and 6 restarts
    assert "Failure to converge to a sufficient solution" in cap.out
    assert abs(gfix.av_plaquette(L.U, d) - lat400["plaquette"]) < 1e-13


def test_coulomb_entry_points_on_a_site_lattice(lib, lat400, capfd):
    """Coulomb_FA (CFACG.c:531-636) and Coulomb (Coulomb.c:32-106) on
    lat[i].O[mu] equal the flat solve; Coulomb reports the initial and
    final link traces and plaquette."""
    d = _dims(lat400)
    set_latt(lib, d, gf_alpha=0.09)
    L = SiteLattice(lat400["links"])
    it = lib.Coulomb_FA(L.sites, None, 1e-14, 650, 1)
    flat = gfix.coulomb_fix(lat400["links"], d, 0.09, 1e-14, 650, "FACG")
    assert it == flat.iters
    assert np.array_equal(L.U, flat.links)
    L2 = SiteLattice(lat400["links"])
    it2 = lib.Coulomb(L2.sites, 1e-14, 650)
    flush_c_stdio()
    out = capfd.readouterr().out
    assert it2 == flat.iters
    assert np.array_equal(L2.U, gfix.latt_reunitU(flat.links, d))
    pl = [float(x) for x in re.findall(r"\[GF\] Plaquette :: ([0-9.]+)", out)]
    assert len(pl) == 2 and all(abs(p - lat400["plaquette"]) < 1e-13 for p in pl)
    assert f"Iterations :: {it2} ||" in out


@pytest.fixture(scope="module")
def hb24x16():
    """A 24^3x16 heatbath configuration: 221184 sites, 3.4 staging chunks
    of 65536 sites (every slot of the ring of three used, one reused, the
    last chunk short)."""
    from glu_b200.workload import heatbath_config
    d = (24, 24, 24, 16)
    return d, heatbath_config(d, seed=5, iterations=30, beta=6.0, n_or=4)


def test_chunked_staging_of_a_large_site_lattice(lib, hb24x16, capfd):
    """The links travel between lat[i].O[mu] and the device in chunks
    through pinned buffers (gather of one chunk overlapping the copy of the
    last): Landau, FACG, Coulomb_FA and Coulomb on a lattice of several
    chunks return, bit for bit, what the flat entry points return for the
    same contiguous links."""
    d, U = hb24x16
    set_latt(lib, d, gf_alpha=0.08, seed=3)
    L = SiteLattice(U)
    it = lib.Landau(L.sites, 1e-12, 3000, b"unused")
    ref = gfix.landau_driver(U, d, 0.08, 1e-12, 3000, restart_seed=3)
    assert it == ref.iters != GLU_FAILURE
    assert np.array_equal(L.U, ref.links)
    L = SiteLattice(U)
    th = C.c_double(0.0)
    it = lib.FACG(L.sites, None, C.byref(th), 1e-12, 3000)
    flat = gfix.landau_fix(U, d, 0.08, 1e-12, 3000, "FACG")
    assert it == flat.iters and th.value == flat.theta
    assert np.array_equal(L.U, flat.links)
    set_latt(lib, d, gf_alpha=0.09)
    L = SiteLattice(U)
    it = lib.Coulomb_FA(L.sites, None, 1e-12, 3000, 1)
    flat = gfix.coulomb_fix(U, d, 0.09, 1e-12, 3000, "FACG")
    assert it == flat.iters
    assert np.array_equal(L.U, flat.links)
    L = SiteLattice(U)
    it = lib.Coulomb(L.sites, 1e-12, 3000)
    _, fin = gfix.coulomb_driver(U, d, 0.09, 1e-12, 3000)
    assert it == fin.iters
    assert np.array_equal(L.U, fin.links)
    flush_c_stdio()
    capfd.readouterr()


# --- GLU's own program, relinked ------------------------------------------




def _run(binary, tmp_path, gftype, tune, tag):
    d = (4, 4, 4, 8)
    inp = tmp_path / f"in_{gftype}"
    inp.write_text(INPUT.format(d0=d[0], d1=d[1], d2=d[2], d3=d[3], gftype=gftype,
                                tune=tune, max_iters=650))
    out = tmp_path / f"{tag}_{gftype}.nersc"
    env = dict(os.environ, OMP_NUM_THREADS="4")
    p = subprocess.run([str(binary), "-i", str(inp), "-c", str(GOLDEN / "lat400.nersc"),
                        "-o", str(out)], cwd=tmp_path, env=env, capture_output=True,
                       text=True, timeout=600)
    return p, out


@pytest.mark.parametrize("gftype, tune", [("LANDAU", 0.08), ("COULOMB", 0.09)])
def test_relinked_glu_program_runs_the_gpu_path(reference, tmp_path, gftype, tune):
    """GLU's program linked with libglu_gfix.so ahead of its own objects
    (oracle/Makefile `relink`): same exit code, "[GF]" report and written
    configuration as the stock program, within GLU's convergence freedom."""
    stock = ROOT / "oracle" / "_ref" / "glu"
    gpu = ROOT / "oracle" / "_ref" / "glu_gpu"
    if not (stock.exists() and gpu.exists()):
        pytest.skip("oracle/_ref/glu or glu_gpu not built")
    p_ref, f_ref = _run(stock, tmp_path, gftype, tune, "ref")
    p_gpu, f_gpu = _run(gpu, tmp_path, gftype, tune, "gpu")
    assert p_ref.returncode == 0, p_ref.stderr[-2000:]
    assert p_gpu.returncode == 0, p_gpu.stderr[-2000:]
    assert f_ref.exists() and f_gpu.exists()

    def plaq(text):
        return [float(x) for x in re.findall(r"\[GF\] Plaquette :: ([0-9.]+)", text)]

    def iters(text):
        # Landau: output_fixing_info's count; Coulomb: the total that
        # Coulomb() prints after the per-slice lines of Coulomb_FA
        m = re.search(r"\[GF\] Iters :: (\d+)", text) or \
            re.search(r"\[GF\] Tuning :: [0-9.]+ \|\| Iterations :: (\d+)", text)
        return int(m.group(1))

    pr, pg = plaq(p_ref.stdout), plaq(p_gpu.stdout)
    assert len(pr) == len(pg) > 0
    assert np.allclose(pr, pg, rtol=0, atol=1e-13)
    tol = 3 if gftype == "LANDAU" else 12
    assert abs(iters(p_gpu.stdout) - iters(p_ref.stdout)) <= tol
    # the written configurations, read back with GLU's own reader
    U_ref = reference.read_file(f_ref)
    U_gpu = reference.read_file(f_gpu)
    assert abs(reference.plaquette() - pr[-1]) < 1e-13
    # both at theta < 1e-14 in the same Gribov copy: the links agree to the
    # freedom the stopping rule leaves (a few ulp-scale iterations apart)
    assert np.abs(U_gpu - U_ref).max() < 1e-6
    if gftype == "LANDAU":
        # GLU's own theta_test_lin on the GPU-fixed configuration
        assert reference.theta_test_lin() < 1e-13


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_relinked_program_at_the_headline_shape(headline_config, tmp_path, precision):
    """GLU's relinked program on the 32^3x64 benchmark configuration (the
    links written as a NERSC 3x3 file, which GLU reads back exactly):
    Landau() reports the iteration count, plaquette and functional of
    gfix_landau_driver on the same links.  The wall time of the call --
    GLU's own [TIMER] around Landau(), which covers whatever of the device
    context's creation the configuration's read did not hide, the
    workspaces, the gather and scatter of GLU's site lattice and the solve
    -- is printed beside gfix_landau_driver's end-to-end time (pinned host
    links, warm engine), with the phases of the call (GLU_GFIX_TIMING)."""
    from glu_b200 import nersc
    from glu_b200._lib import GfixParams, GfixResult, check
    gpu = ROOT / "oracle" / "_ref" / "glu_gpu"
    if not gpu.exists():
        pytest.skip("oracle/_ref/glu_gpu not built")
    d = (32, 32, 32, 64)
    cfg = tmp_path / "hb.nersc"
    nersc.write(cfg, headline_config, d, datatype="4D_SU3_GAUGE_3x3")
    inp = tmp_path / "in"
    inp.write_text(INPUT.format(d0=d[0], d1=d[1], d2=d[2], d3=d[3], gftype="LANDAU",
                                tune=0.08, max_iters=4000))
    env = dict(os.environ, GLU_GFIX_TIMING="1", GLU_GFIX_PRECISION=precision)
    p = subprocess.run([str(gpu), "-i", str(inp), "-c", str(cfg)], cwd=tmp_path,
                       env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    out = p.stdout
    # [TIMER] lines: the read of the configuration, then Landau()
    timers = [float(x) for x in re.findall(r"\[TIMER\] elapsed :: ([0-9.e+-]+) s", out)]
    assert len(timers) >= 2
    t_call = timers[1]
    phases = re.search(r"\[GF\] GPU timing(.*)", out).group(1)
    it = int(re.search(r"\[GF\] Iters :: (\d+)", out).group(1))
    plaq = float(re.findall(r"\[GF\] Plaquette :: ([0-9.]+)", out)[-1])
    func = float(re.search(r"\[GF\] Functional :: ([0-9.]+)", out).group(1))

    # the same fix through the flat driver: pinned host links, warm engine
    lib = _lib.load()
    V = int(np.prod(d))
    host = torch.from_numpy(headline_config.view(np.float64).reshape(-1)).pin_memory()
    work = torch.empty_like(host).pin_memory()
    cd = (C.c_size_t * 4)(*d)
    prm = GfixParams()
    prm.gf_alpha, prm.accuracy, prm.max_iters = 0.08, 1e-14, 4000
    prm.precision = 1 if precision == "MIXED" else 0
    prm.switch_theta = 1e-9
    prm.max_restarts, prm.restart_seed = 6, 0
    r = GfixResult()
    obs, dg = np.zeros(3), np.zeros(6)
    dp = C.POINTER(C.c_double)
    times = []
    for _ in range(3):
        work.copy_(host)
        t0 = time.perf_counter()
        check(lib.gfix_landau_driver(work.data_ptr(), cd, C.byref(prm), C.byref(r),
                                     obs.ctypes.data_as(dp), dg.ctypes.data_as(dp)))
        times.append(time.perf_counter() - t0)
    assert it == r.iters
    assert abs(plaq - obs[2]) < 1e-13
    assert abs(func - obs[1]) < 1e-12
    print("\n[%s] Landau() in GLU's program %.3f s (%d iterations;%s); "
          "gfix_landau_driver end to end %.3f s (best of %d after the first %.3f s)"
          % (precision, t_call, it, phases, min(times[1:]), len(times) - 1, times[0]))


def test_relinked_program_coulomb_at_the_headline_shape(headline_config, tmp_path):
    """GLU's relinked program fixing every time slice of the 32^3x64
    benchmark configuration to Coulomb gauge through Coulomb() (FP64): the
    reported iteration total and final plaquette equal gfix_coulomb_driver's
    on the same links; GLU's [TIMER] around the call is printed beside the
    flat driver's end-to-end time, with the phases of the call."""
    from glu_b200 import nersc
    from glu_b200._lib import GfixParams, GfixResult, check
    gpu = ROOT / "oracle" / "_ref" / "glu_gpu"
    if not gpu.exists():
        pytest.skip("oracle/_ref/glu_gpu not built")
    d = (32, 32, 32, 64)
    cfg = tmp_path / "hb.nersc"
    nersc.write(cfg, headline_config, d, datatype="4D_SU3_GAUGE_3x3")
    inp = tmp_path / "in"
    inp.write_text(INPUT.format(d0=d[0], d1=d[1], d2=d[2], d3=d[3], gftype="COULOMB",
                                tune=0.08, max_iters=4000))
    env = dict(os.environ, GLU_GFIX_TIMING="1")
    p = subprocess.run([str(gpu), "-i", str(inp), "-c", str(cfg)], cwd=tmp_path,
                       env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    out = p.stdout
    timers = [float(x) for x in re.findall(r"\[TIMER\] elapsed :: ([0-9.e+-]+) s", out)]
    assert len(timers) >= 2
    phases = re.search(r"\[GF\] GPU timing(.*)", out).group(1)
    it = int(re.search(r"\[GF\] Tuning :: [0-9.]+ \|\| Iterations :: (\d+)", out).group(1))
    plaq = float(re.findall(r"\[GF\] Plaquette :: ([0-9.]+)", out)[-1])

    lib = _lib.load()
    host = torch.from_numpy(headline_config.view(np.float64).reshape(-1)).pin_memory()
    work = torch.empty_like(host).pin_memory()
    cd = (C.c_size_t * 4)(*d)
    prm = GfixParams()
    prm.gf_alpha, prm.accuracy, prm.max_iters = 0.08, 1e-14, 4000
    r = GfixResult()
    o0, g0, o1, g1 = np.zeros(3), np.zeros(6), np.zeros(3), np.zeros(6)
    dp = C.POINTER(C.c_double)
    times = []
    for _ in range(2):
        work.copy_(host)
        t0 = time.perf_counter()
        check(lib.gfix_coulomb_driver(work.data_ptr(), cd, C.byref(prm), C.byref(r),
                                      o0.ctypes.data_as(dp), g0.ctypes.data_as(dp),
                                      o1.ctypes.data_as(dp), g1.ctypes.data_as(dp)))
        times.append(time.perf_counter() - t0)
    assert it == r.iters
    assert abs(plaq - o1[2]) < 1e-13
    print("\n[COULOMB] Coulomb() in GLU's program %.3f s (%d slice iterations;%s); "
          "gfix_coulomb_driver end to end %.3f s (after a first call of %.3f s)"
          % (timers[1], it, phases, times[1], times[0]))
