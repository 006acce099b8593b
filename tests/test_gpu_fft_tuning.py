"""FFT plans: the default plan per shape and the autotuned ones
(gfix_fft_tuning) give the same transforms and the same fixes up to
rounding.  Through the C ABI."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402


@pytest.fixture
def tuned():
    gfix.fft_tuning(True)
    try:
        yield
    finally:
        gfix.fft_tuning(False)


def test_default_plan_is_compile_time_for_common_shapes():
    (xy, b, zt), ms = gfix.fft_plan((32, 32, 32, 64))
    assert xy == -1 and zt == -1 and b == 4 and ms == (0.0, 0.0)
    (xy, b, zt), _ = gfix.fft_plan((6, 10, 5, 3))  # radix 5: generic passes
    assert xy >= 0 and zt >= 0


@pytest.mark.parametrize("dims,ndim", [((8, 8, 16, 32), 4), ((12, 6, 10, 6), 4),
                                       ((16, 8, 32, 2), 3)])
def test_tuned_transform_matches_oracle(oracle, tuned, dims, ndim):
    rng = np.random.default_rng(4)
    n = int(np.prod(dims[:ndim]))
    f = rng.normal(size=(4, n)) + 1j * rng.normal(size=(4, n))
    got = gfix.fourier_accelerate(f, dims, ndim)
    ref = oracle.fourier_accelerate(f, dims, ndim)
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()
    plan, ms = gfix.fft_plan(dims, coulomb=(ndim == 3))
    assert ms[0] > 0 and ms[1] > 0 and plan[1] >= 1


def test_tuned_fix_reaches_accuracy(hb8, tuned):
    d = tuple(int(x) for x in hb8["dims"])
    r = gfix.landau_fix(hb8["links"], d, 0.08, 1e-14, 1000)
    assert r.theta < 1e-14
    assert abs(r.iters - int(hb8["landau_facg_iters"])) <= 10
    _, _, p0 = gfix.observables(hb8["links"], d)
    _, _, p1 = gfix.observables(r.links, d)
    assert abs(p1 - p0) < 1e-13
