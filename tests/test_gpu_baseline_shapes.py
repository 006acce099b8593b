"""Parity at the lattice shapes the benchmarks run on.

The FFT passes are compile-time specialised per extent (fft_ct.cuh), so each
benchmark shape runs its own kernels: the 4D transform at 16^3x32 and
24^3x48 (the ensemble), 32^3x64 (the headline) and 48^3x96, and the 3D slice
transform at 16^3, 24^3, 48^3 and 64^3 (Coulomb).  Each is compared with the
oracle's FFTW-convention transform.  At 32^3x64 the Landau FACG trajectory of
the headline's first configuration (a beta 6.0 heatbath configuration made on
the GPU) is compared with GLU itself (oracle/_ref, run live), and the links
after a few iterations with the oracle.  All calls go through the C ABI.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402

HEADLINE = (32, 32, 32, 64)


def _fields(n, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(4, n)) + 1j * rng.normal(size=(4, n))


@pytest.mark.parametrize("dims", [(16, 16, 16, 32), (24, 24, 24, 48),
                                  HEADLINE, (48, 48, 48, 96)],
                         ids=lambda d: "x".join(map(str, d)))
def test_fourier_accelerate_at_benchmark_shapes(oracle, dims):
    """FOURIER_ACCELERATE3 with the default plan the solver uses."""
    f = _fields(int(np.prod(dims)), 17)
    got = gfix.fourier_accelerate(f, dims)
    ref = oracle.fourier_accelerate(f, dims, 4)
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("dims", [(16, 16, 16, 2), (24, 24, 24, 2),
                                  (48, 48, 48, 2), (64, 64, 64, 2)],
                         ids=lambda d: "x".join(map(str, d[:3])))
def test_fourier_accelerate2_at_benchmark_slices(oracle, dims):
    """FOURIER_ACCELERATE2 on one time slice of the Coulomb lattices."""
    f = _fields(dims[0] * dims[1] * dims[2], 18)
    got = gfix.fourier_accelerate(f, dims, 3)
    ref = oracle.fourier_accelerate(f, dims, 3)
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


def test_headline_links_match_oracle_after_two_iterations(oracle, headline_config):
    """Links after exactly two FACG iterations (SD start, then CG) at the
    headline shape, against the oracle, at the same iteration count."""
    U = headline_config
    r = gfix.landau_fix(U, HEADLINE, 0.08, 1e-30, 2, "FACG")
    o = oracle.landau(U, HEADLINE, 0.08, 1e-30, 2, "FACG")
    assert r.iters == o["iters"] == gfix.SENTINEL
    assert abs(r.theta - o["theta"]) < 1e-11 * o["theta"]
    # the largest of 7.5e7 entry differences: a few ulp of O(1) entries
    assert np.abs(r.links - o["links"]).max() < 1e-12


def test_headline_trajectory_matches_reference(reference, headline_config):
    """The first 20 FACG iterations at 32^3x64 against GLU run live: theta
    and the gauge functional at every derivative evaluation of GLU on one
    thread (the instrumented build records its trajectory single-threaded).
    GLU does not reproduce itself beyond summation order, so its spread is
    measured too: the theta after k iterations on all host threads, at
    every fourth k.  The bound is 1e-10 relative where that spread is below
    1e-10, and 100x the spread beyond."""
    U = headline_config
    n = 20
    r = gfix.landau_fix(U, HEADLINE, 0.08, 1e-30, n, "FACG", traj_cap=n + 4)
    reference.setup(HEADLINE, 1, 0.08)
    reference.put_links(U)
    ref = reference.landau_fa(1e-30, n, "FACG", traj_cap=n + 4)
    m = min(len(ref["traj_theta"]), len(r.traj_theta))
    assert m == n + 1  # the SD start, then one per CG iteration
    th, th_ref = r.traj_theta[:m], ref["traj_theta"][:m]
    fn, fn_ref = r.traj_func[:m], ref["traj_func"][:m]
    # GLU's spread: theta of its k-iteration runs on many threads (entry k
    # of the trajectory is the theta measured at the top of iteration k)
    reference.set_threads(max(2, min(16, os.cpu_count() or 2)))
    env = np.zeros(m)
    for k in range(4, n + 1, 4):
        reference.put_links(U)
        tk = reference.landau_fa(1e-30, k, "FACG")["theta"]
        env[k] = abs(tk - th_ref[k])
    reference.set_threads(1)
    # between samples the spread is taken as the next sample's (it grows)
    for k in range(m - 1, 0, -1):
        if env[k] == 0 and k + 1 < m:
            env[k] = env[k + 1]
    rel_env = env / th_ref
    bad = np.nonzero(rel_env > 1e-10)[0]
    prefix = int(bad[0]) if len(bad) else m
    assert prefix >= 4
    rel = np.abs(th - th_ref) / th_ref
    assert rel[:prefix].max() < 1e-10
    assert np.all(np.abs(th - th_ref) <= 100 * env + 1e-10 * th_ref)
    # the functional is a sum of 2.5e7 link traces: its summation order
    # alone moves it by ~1e-13 at this volume
    assert np.abs(fn[:prefix] - fn_ref[:prefix]).max() < 1e-12
    assert np.abs(fn - fn_ref).max() < 1e-9


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_headline_full_fix_keeps_the_plaquette(headline_config, precision):
    """A complete fix to theta < 1e-14 stays on the input's gauge orbit:
    the average plaquette of the fixed links, reunitarised as GLU's Landau
    driver does before it reports (output_fixing_info), equals the input's
    to 1e-13.  (Unreunitarised links drift off SU(3) over a long fix, by
    GLU's own update, which rebuilds one column per step from the other
    two; the GLU-named Landau() and gfix_landau_driver reunitarise.)"""
    U = headline_config
    plaq = gfix.av_plaquette(U, HEADLINE)
    r = gfix.landau_fix(U, HEADLINE, 0.08, 1e-14, 20000, "FACG",
                        precision=precision)
    assert r.iters != gfix.SENTINEL
    assert r.theta < 1e-14
    fixed = gfix.latt_reunitU(r.links, HEADLINE)
    assert abs(gfix.av_plaquette(fixed, HEADLINE) - plaq) < 1e-13
    d = gfix.landau_driver(U, HEADLINE, 0.08, 1e-14, 20000, precision=precision)
    assert d.iters == r.iters
    assert abs(d.plaquette - plaq) < 1e-13
