"""Landau FA gauge fixing on the GPU against the oracle and the reference.

All calls go through the C ABI (libglu_gfix.so via ctypes)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def _dims(g):
    return tuple(int(d) for d in g["dims"])


def _envelope_prefix(g, tol=1e-10):
    env = _rel(g["landau_facg_env8"],
               g["landau_facg_traj_theta"][1:1 + len(g["landau_facg_env8"])])
    bad = np.nonzero(env > tol)[0]
    return int(bad[0]) + 1 if len(bad) else len(env) + 1


@pytest.mark.parametrize("case", ["lat400", "hb8"])
def test_observables_match_oracle(oracle, case, request):
    g = request.getfixturevalue(case)
    d = _dims(g)
    th, fn, pl = gfix.observables(g["links"], d)
    assert abs(th - oracle.theta_test_lin(g["links"], d)) < 1e-12 * th
    assert abs(fn - g["functional"]) < 1e-14
    assert abs(pl - g["plaquette"]) < 1e-13


@pytest.mark.parametrize("dims", [(4, 4, 4, 8), (8, 6, 4, 12), (6, 10, 5, 3),
                                  (8, 8, 48, 96), (8, 8, 32, 64)])
def test_fourier_accelerate_matches_oracle(oracle, dims):
    rng = np.random.default_rng(7)
    V = int(np.prod(dims))
    f = rng.normal(size=(4, V)) + 1j * rng.normal(size=(4, V))
    got = gfix.fourier_accelerate(f, dims)
    ref = oracle.fourier_accelerate(f, dims, 4)
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("dims", [(4, 4, 4, 8), (16, 8, 32, 2), (6, 10, 5, 3),
                                  (16, 16, 64, 2), (16, 16, 48, 2)])
def test_fourier_accelerate3_matches_oracle(oracle, dims):
    """FOURIER_ACCELERATE2 (one time slice, MAX_COULOMB / p^2 in 3D)."""
    rng = np.random.default_rng(8)
    n = dims[0] * dims[1] * dims[2]
    f = rng.normal(size=(4, n)) + 1j * rng.normal(size=(4, n))
    got = gfix.fourier_accelerate(f, dims, 3)
    ref = oracle.fourier_accelerate(f, dims, 3)
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("which", ["input", "landau", "coulomb"])
def test_link_diagnostics_match_reference(lat400, which):
    """all_links, indivlinks and both const_time definitions of GLU (fixture
    values from the reference build) on the input and on the fixed links."""
    g = lat400
    links = {"input": g["links"], "landau": g["landau_facg_links"],
             "coulomb": g["coulomb_facg_links"]}[which]
    ref = g[f"diag_{which}"]
    got = gfix.link_diagnostics(links, _dims(g))
    assert abs(got["splink"] - ref[0]) < 1e-14
    assert abs(got["tlink"] - ref[1]) < 1e-14
    assert abs(got["link"] - ref[3]) < 1e-14
    # GLU prints the maximum trace divided by NC
    assert abs(got["link_max"] - ref[4] / 3.0) < 1e-14
    # a difference of slice sums of O(1) entries: rounding floor ~1e-15
    assert abs(got["const_lin"] - ref[5]) <= 1e-12 * ref[5] + 1e-15
    # the same with the exact logarithm of every temporal link
    assert abs(got["const_log"] - ref[6]) <= 1e-11 * ref[6] + 1e-13


def test_reunit_matches_oracle(oracle, lat400):
    g = lat400
    rng = np.random.default_rng(1)
    U = g["links"] + 1e-3 * (rng.normal(size=g["links"].shape)
                             + 1j * rng.normal(size=g["links"].shape))
    got = gfix.latt_reunitU(U, _dims(g))
    ref = oracle.reunit(U)
    assert np.abs(got - ref).max() < 1e-14


@pytest.mark.parametrize("case", ["lat400", "hb8"])
def test_landau_facg_matches_reference(case, request):
    g = request.getfixturevalue(case)
    d = _dims(g)
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 650, "FACG", traj_cap=5000)
    ref = g["landau_facg_traj_theta"]
    n = _envelope_prefix(g)
    # theta to 1e-10 relative wherever the reference reproduces itself to
    # 1e-10 across OpenMP thread counts
    assert _rel(r.traj_theta[:n], ref[:n]).max() < 1e-10
    assert np.abs(r.traj_func[:n] - g["landau_facg_traj_func"][:n]).max() < 1e-13
    # beyond it, within 100x the reference's own spread
    m = min(len(g["landau_facg_env8"]), len(r.traj_theta) - 1, len(ref) - 1)
    env = np.abs(g["landau_facg_env8"][:m] - ref[1:1 + m])
    assert np.all(np.abs(r.traj_theta[1:1 + m] - ref[1:1 + m])
                  <= 100 * env + 1e-10 * ref[1:1 + m])
    assert abs(r.iters - int(g["landau_facg_iters"])) <= 3
    assert r.theta < 1e-14
    # gauge invariance: plaquette unchanged
    assert abs(gfix.av_plaquette(r.links, d) - g["plaquette"]) < 1e-13


def test_landau_fasd_fixed_step_matches_reference(lat400):
    """GLU_GFIX_SD semantics: no line search, the whole run agrees."""
    g = lat400
    d = _dims(g)
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 650, "FASD",
                        sd_fixed_step=True, traj_cap=5000)
    ref = g["landau_fasd_sd_traj_theta"]
    assert r.iters == int(g["landau_fasd_sd_iters"])
    assert _rel(r.traj_theta[: len(ref)], ref).max() < 1e-9
    # links at the same iteration count
    assert np.abs(r.links - g["landau_fasd_sd_links"]).max() < 1e-12


def test_landau_fasd_line_search_matches_reference(lat400):
    g = lat400
    d = _dims(g)
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 650, "FASD", traj_cap=5000)
    ref = g["landau_fasd_ls_traj_theta"]
    assert _rel(r.traj_theta[:20], ref[:20]).max() < 1e-10
    assert abs(r.iters - int(g["landau_fasd_ls_iters"])) <= 10
    assert r.theta < 1e-14


def test_landau_matches_oracle_step_by_step(oracle, lat400):
    """Iteration-count-matched links against the oracle for a short run
    (acc 1e-30 never converges; both stop after exactly k iterations)."""
    g = lat400
    d = _dims(g)
    for k in (1, 2, 5):
        r = gfix.landau_fix(g["links"], d, 0.08, 1e-30, k, "FACG")
        o = oracle.landau(g["links"], d, 0.08, 1e-30, k, "FACG")
        assert r.iters == o["iters"] == gfix.SENTINEL
        assert abs(r.theta - o["theta"]) < 1e-12 * o["theta"]
        assert np.abs(r.links - o["links"]).max() < 1e-13


def test_mixed_precision_reaches_fp64_accuracy(hb8):
    g = hb8
    d = _dims(g)
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 2000, "FACG",
                        precision="MIXED", switch_theta=1e-9)
    assert r.iters != gfix.SENTINEL
    assert r.theta < 1e-14
    assert r.iters_fp32 > 0
    # the links stay on the gauge orbit of the input to FP64 accuracy
    assert abs(gfix.av_plaquette(r.links, d) - g["plaquette"]) < 1e-13
    th, fn, _ = gfix.observables(r.links, d)
    assert th < 1e-13
    # same Landau-gauge functional as the FP64 solve (same Gribov region)
    r64 = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 2000, "FACG")
    assert abs(fn - gfix.gauge_functional(r64.links, d)) < 1e-8


def test_mixed_precision_on_a_thermalised_configuration(monkeypatch):
    """A genuine beta 6.0 heatbath configuration (16^3x32, generated on the
    GPU): theta crosses a plateau, on which the FP32 phase hands over by the
    stall rule; both the default rule and the threshold-only switch reach
    theta < 1e-14 on the input's gauge orbit."""
    from glu_b200.workload import heatbath_config
    d = (16, 16, 16, 32)
    U = heatbath_config(d, seed=7, iterations=300)
    plaq = gfix.av_plaquette(U, d)
    for stall in (None, "0"):
        if stall is None:
            monkeypatch.delenv("GLU_GFIX_STALL", raising=False)
        else:
            monkeypatch.setenv("GLU_GFIX_STALL", stall)
        r = gfix.landau_fix(U, d, 0.08, 1e-14, 20000, "FACG", precision="MIXED",
                            switch_theta=1e-9)
        assert r.iters != gfix.SENTINEL
        assert r.theta < 1e-14
        assert 0 < r.iters_fp32 < r.iters
        assert abs(gfix.av_plaquette(r.links, d) - plaq) < 1e-12
        assert gfix.observables(r.links, d)[0] < 1e-13


def test_nonconvergence_sentinel(lat400):
    g = lat400
    r = gfix.landau_fix(g["links"], _dims(g), 0.08, 1e-14, 4, "FACG")
    assert r.iters == gfix.SENTINEL


def test_already_fixed_returns_zero(lat400):
    g = lat400
    d = _dims(g)
    fixed = g["landau_facg_links"]
    r = gfix.landau_fix(fixed, d, 0.08, 1e-10, 100, "FACG")
    assert r.iters == 0


def test_random_odd_lattice_against_oracle(oracle):
    """Extents with radix-3 and radix-5 factors and an odd extent."""
    from glu_b200.workload import random_su3
    d = (6, 5, 4, 3)
    V = int(np.prod(d))
    rng = np.random.default_rng(11)
    U = random_su3(V * 4, rng).reshape(V, 4, 3, 3)
    # a smooth-ish config: mix with the identity and reunitarise
    U = oracle.reunit(np.eye(3) + 0.3 * U)
    r = gfix.landau_fix(U, d, 0.08, 1e-30, 3, "FACG", traj_cap=10)
    o = oracle.landau(U, d, 0.08, 1e-30, 3, "FACG", traj_cap=10)
    ot = o["traj_theta"]
    # theta falls by six decades in three steps here: compare against the
    # scale of the run, not of the tiny last value
    assert np.all(np.abs(r.traj_theta - ot) <= 1e-11 * ot + 1e-14 * ot[0])
    assert np.abs(r.links - o["links"]).max() < 1e-12


@pytest.mark.parametrize("case, which", [("lat400", "links"),
                                         ("lat400", "landau_facg_links"),
                                         ("lat400", "coulomb_facg_links"),
                                         ("hb8", "links")])
def test_gf_check_matches_reference(reference, case, which, request):
    """GLU's gf_check numbers (theta_test_lin and theta_test_log with their
    largest local values, over four and three directions, and const_time)
    against GLU itself on the same links.  On fixed links theta is a sum of
    squares of rounding-sized derivatives, so the comparison there is
    relative to GLU's own rounding (1e-6), elsewhere 1e-12."""
    g = request.getfixturevalue(case)
    d = _dims(g)
    U = g[which]
    got = gfix.gf_check(U, d)
    reference.setup(d, 1, 0.08)
    reference.put_links(U)
    ref = reference.gf_check()
    keys = ["landau_lin", "landau_lin_max", "landau_log", "landau_log_max",
            "const_lin", "const_log", "coulomb_lin", "coulomb_lin_max",
            "coulomb_log", "coulomb_log_max"]
    for k, r in zip(keys, ref):
        tol = 1e-6 if r < 1e-8 else 1e-11
        # const_time is a difference of slice sums of O(1) entries: its
        # rounding floor is ~1e-15 absolute
        floor = 1e-15 if k.startswith("const") else 1e-300
        assert abs(got[k] - r) <= tol * abs(r) + floor, (k, got[k], r)
    text = gfix.gf_check_report(got)
    assert "[GFACC LANDAU]      LOG ::" in text and "[GFACC MAX COULOMB] LOG ::" in text
