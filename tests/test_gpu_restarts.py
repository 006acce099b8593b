"""Random restarts of a failed Landau fix (GLU's Landau driver,
src/Gfix/Landau.c:303-340) through gfix_landau with max_restarts > 0.

GLU re-reads its input after a failed FACG, applies a random gauge
transform (random_transform, src/Geometry/random_config.c:107-120) and
solves again, at most GF_GLU_FAILURES - 1 = 6 times.  Its iteration count
keeps the first attempt's sentinel and adds max_iters per failed restart and
the successful attempt's count; GLU_FAILURE when every attempt failed.  The
transforms come from this library's own generator, so restarted runs are
compared with GLU's accounting and with gauge invariance, not value for
value.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402

GLU_FAILURE = (1 << 64) - 1


def _dims(g):
    return tuple(int(d) for d in g["dims"])


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_every_attempt_fails(hb8, precision):
    g = hb8
    d = _dims(g)
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 4, "FACG", precision=precision,
                        max_restarts=6, restart_seed=11)
    assert r.iters == GLU_FAILURE
    assert r.restarts == 6
    # the last attempt's links: a gauge transform of the input plus four
    # iterations, on the input's gauge orbit
    assert abs(gfix.av_plaquette(r.links, d) - g["plaquette"]) < 1e-13
    # restarts start from a random point of the orbit, not from the input
    r0 = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 4, "FACG", precision=precision)
    assert r0.iters == gfix.SENTINEL and r0.restarts == 0
    assert np.abs(r.links - r0.links).max() > 1e-2


def test_restarts_are_reproducible(hb8):
    g = hb8
    d = _dims(g)
    a = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 6, "FACG", max_restarts=2,
                        restart_seed=3)
    b = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 6, "FACG", max_restarts=2,
                        restart_seed=3)
    c = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 6, "FACG", max_restarts=2,
                        restart_seed=4)
    assert np.array_equal(a.links, b.links)
    assert not np.array_equal(a.links, c.links)


def test_a_restart_converges_where_the_first_attempt_failed(hb8):
    """With max_iters below what the input needs, the first attempt fails;
    the random restarts start elsewhere on the gauge orbit, and one of them
    converges within max_iters.  The count is GLU's: sentinel + max_iters x
    (restarts - 1) + the successful attempt's count."""
    g = hb8
    d = _dims(g)
    n0 = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 5000, "FACG").iters
    found = None
    for m in range(max(n0 - 40, 10), n0, 4):
        first = gfix.landau_fix(g["links"], d, 0.08, 1e-14, m, "FACG")
        if first.iters != gfix.SENTINEL:
            continue  # converged (or continued) within m: no restart needed
        for seed in range(1, 7):
            r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, m, "FACG",
                                max_restarts=6, restart_seed=seed)
            assert abs(gfix.av_plaquette(r.links, d) - g["plaquette"]) < 1e-13
            if r.iters == GLU_FAILURE:
                assert r.restarts == 6
                continue
            assert 1 <= r.restarts <= 6
            k = r.iters - gfix.SENTINEL - m * (r.restarts - 1)
            assert 0 < k <= m
            assert r.theta < 1e-14
            assert gfix.theta_test_lin(r.links, d) < 1e-13
            found = (m, seed, r.restarts, k)
            break
        if found:
            break
    assert found is not None, "no restart converged"


def test_luxury_copies(hb8):
    """GLU's luxury_copy_fast (LUXURY_GAUGE, src/Gfix/Landau.c:92-211):
    random gauge copies fixed to 1e-6, one kept -- the largest functional by
    default, the smallest under BEST_COPY -- then fixed to the accuracy.
    With the same seed both rules choose among the same copies, so the
    BEST_COPY result's functional is not above the default's."""
    g = hb8
    d = _dims(g)
    runs = {}
    for best in (False, True):
        r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 2000, "FACG",
                            luxury_copies=4, luxury_best=best, restart_seed=9)
        assert r.iters != gfix.SENTINEL and r.iters > 0
        assert r.theta < 1e-14
        fixed = gfix.latt_reunitU(r.links, d)
        assert abs(gfix.av_plaquette(fixed, d) - g["plaquette"]) < 1e-13
        runs[best] = gfix.gauge_functional(r.links, d)
    assert runs[True] <= runs[False] + 1e-9
    # the copies start from random points of the orbit: the kept copy is
    # not the plain fix of the input
    plain = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 2000, "FACG")
    r = gfix.landau_fix(g["links"], d, 0.08, 1e-14, 2000, "FACG",
                        luxury_copies=1, restart_seed=9)
    assert np.abs(r.links - plain.links).max() > 1e-3
