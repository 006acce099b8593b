"""Batches of configurations (gfix_batch_*): every configuration of a batch
must come out exactly as from its own gfix_landau call -- the batch runs
each configuration's kernel sequence unchanged, only concurrently, with
converged configurations masked out.  Sequences (gfix_landau_sequence) the
same, one configuration after another with overlapped copies.  All calls go
through the C ABI."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402
from glu_b200._lib import GfixError  # noqa: E402
from glu_b200.workload import random_su3, tiled_config  # noqa: E402


def _dims(g):
    return tuple(int(d) for d in g["dims"])


def _transformed(U, dims, seed):
    """U under a seeded random gauge transformation (same orbit)."""
    rng = np.random.default_rng(seed)
    V = U.shape[0]
    g = random_su3(V, rng)
    Lx, Ly, Lz, Lt = dims
    idx = np.arange(V).reshape(Lt, Lz, Ly, Lx)
    out = np.empty_like(U)
    for mu, ax in enumerate((3, 2, 1, 0)):
        fwd = np.roll(idx, -1, axis=ax).reshape(V)
        out[:, mu] = g @ U[:, mu] @ np.conj(np.swapaxes(g[fwd], -1, -2))
    return out


@pytest.fixture(scope="module")
def configs(lat400, hb8):
    d4 = _dims(lat400)
    d8 = _dims(hb8)
    d16 = (16, 8, 8, 16)
    return [
        (lat400["links"], d4),
        (_transformed(lat400["links"], d4, 5), d4),
        (hb8["links"], d8),
        (tiled_config(d16, seed=7), d16),
        (_transformed(hb8["links"], d8, 9), d8),
    ]


@pytest.mark.parametrize("algo,precision,acc", [("FACG", "FP64", 1e-14),
                                                ("FASD", "FP64", 1e-12),
                                                ("FACG", "MIXED", 1e-14),
                                                ("FASD", "MIXED", 1e-12)])
def test_batch_equals_single_solves(configs, algo, precision, acc):
    kw = dict(gf_alpha=0.08, accuracy=acc, max_iters=4000, algo=algo,
              precision=precision, switch_theta=1e-9)
    got = gfix.landau_batch(configs, **kw)
    assert len(got) == len(configs)
    for (U, d), r in zip(configs, got):
        one = gfix.landau_fix(U, d, **kw)
        assert r.iters == one.iters and r.iters_fp32 == one.iters_fp32
        assert r.theta == one.theta
        assert np.array_equal(r.links, one.links)
        assert r.theta < acc


def test_batch_of_one_and_repeated_runs(lat400):
    d = _dims(lat400)
    a = gfix.landau_batch([(lat400["links"], d)])[0]
    b = gfix.landau_batch([(lat400["links"], d)])[0]
    one = gfix.landau_fix(lat400["links"], d)
    assert a.iters == b.iters == one.iters
    assert np.array_equal(a.links, one.links) and np.array_equal(b.links, one.links)


def test_empty_batch_and_bad_index():
    assert gfix.landau_batch([]) == []
    from glu_b200 import _lib
    import ctypes as C
    lib = _lib.load()
    p, _, _ = gfix._params(0.08, 1e-14, 100, "FACG", False, "FP64", 1e-9, 0)
    b = lib.gfix_batch_create(C.byref(p))
    try:
        r = _lib.GfixResult()
        assert lib.gfix_batch_result(b, 0, C.byref(r)) != 0
        with pytest.raises(GfixError):
            _lib.check(lib.gfix_batch_result(b, 3, C.byref(r)))
    finally:
        lib.gfix_batch_destroy(b)


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_sequence_equals_single_fixes(precision):
    """gfix_landau_sequence on pinned host links (the copies of neighbouring
    configurations then overlap the solves): every configuration exactly as
    its own gfix_landau call -- links bit for bit, iterations, theta -- and
    its links written back to its own array."""
    import ctypes as C
    from glu_b200 import _lib
    from glu_b200._lib import GfixParams, GfixResult, check
    from glu_b200.workload import heatbath_config
    d = (16, 16, 16, 32)
    Us = [heatbath_config(d, seed=s, iterations=40) for s in (11, 12, 13)]
    lib = _lib.load()
    host = [torch.from_numpy(u.view(np.float64).reshape(-1).copy()).pin_memory() for u in Us]
    p = GfixParams()
    p.gf_alpha, p.accuracy, p.max_iters = 0.08, 1e-12, 2000
    p.precision = 1 if precision == "MIXED" else 0
    p.switch_theta = 1e-9
    ptrs = (C.c_void_p * 3)(*[h.data_ptr() for h in host])
    rs = (GfixResult * 3)()
    cd = (C.c_size_t * 4)(*d)
    check(lib.gfix_landau_sequence(ptrs, 3, cd, C.byref(p), rs))
    for U, h, r in zip(Us, host, rs):
        ref = gfix.landau_fix(U, d, 0.08, 1e-12, 2000, "FACG", precision=precision)
        assert r.iters == ref.iters != gfix.SENTINEL
        assert r.theta == ref.theta
        assert np.array_equal(h.numpy().view(np.complex128).reshape(-1, 4, 3, 3), ref.links)
    # pageable arrays through the Python wrapper: the same results
    seq = gfix.landau_sequence(Us[:2], d, 0.08, 1e-12, 2000, precision=precision)
    for U, s in zip(Us[:2], seq):
        ref = gfix.landau_fix(U, d, 0.08, 1e-12, 2000, "FACG", precision=precision)
        assert s.iters == ref.iters and np.array_equal(s.links, ref.links)


def test_sequence_keeps_restart_accounting(hb8):
    """A sequence passes every parameter on: with max_iters below what the
    configurations need and random restarts allowed, each configuration's
    count, restarts and links equal its own gfix_landau call's (GLU's
    accounting: sentinel + max_iters per failed restart + the successful
    count, or GLU_FAILURE)."""
    d = _dims(hb8)
    Us = [hb8["links"], _transformed(hb8["links"], d, 21)]
    seq = gfix.landau_sequence(Us, d, 0.08, 1e-14, 40, max_restarts=3, restart_seed=7)
    for U, s in zip(Us, seq):
        ref = gfix.landau_fix(U, d, 0.08, 1e-14, 40, "FACG", max_restarts=3,
                              restart_seed=7)
        assert ref.iters != gfix.SENTINEL
        assert (s.iters, s.restarts) == (ref.iters, ref.restarts)
        assert np.array_equal(s.links, ref.links)
