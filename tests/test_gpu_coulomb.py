"""Coulomb FA gauge fixing on the GPU against the oracle and the reference.

The reference (src/Gfix/CFACG.c:531-636) fixes the time slices one after the
other; the GPU fixes all of them in one batched launch sequence.  Its
trajectory comes back slice-major (stride traj_cap / Lt, NaN-padded), the
reference's and the oracle's as one concatenation, so trajectories are
compared slice by slice.  All calls go through the C ABI."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix  # noqa: E402

ACC = 1e-14


def _dims(g):
    return tuple(int(d) for d in g["dims"])


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def _gpu_slices(r, T):
    per = len(r.traj_theta) // T
    rows = r.traj_theta.reshape(T, per)
    return [row[~np.isnan(row)] for row in rows]


def _split(traj, counts):
    out, o = [], 0
    for c in counts:
        out.append(traj[o:o + c])
        o += c
    return out


def _smooth_links(dims, eps, seed):
    """Links near a gauge transform of the identity: reunit(1 + eps X) then a
    random gauge rotation, so that every slice converges in few steps."""
    rng = np.random.default_rng(seed)
    V = int(np.prod(dims))
    X = rng.normal(size=(V, 4, 3, 3)) + 1j * rng.normal(size=(V, 4, 3, 3))
    U = np.eye(3) + eps * X
    U, _ = np.linalg.qr(U)
    U /= np.linalg.det(U)[..., None, None] ** (1.0 / 3.0)
    G, _ = np.linalg.qr(rng.normal(size=(V, 3, 3)) + 1j * rng.normal(size=(V, 3, 3)))
    G /= np.linalg.det(G)[..., None, None] ** (1.0 / 3.0)
    Lx, Ly, Lz, Lt = dims
    idx = np.arange(V).reshape(Lt, Lz, Ly, Lx)
    out = np.empty_like(U)
    for mu, ax in enumerate((3, 2, 1, 0)):
        fwd = np.roll(idx, -1, axis=ax).reshape(V)
        out[:, mu] = G @ U[:, mu] @ np.conj(np.swapaxes(G[fwd], -1, -2))
    return out


def test_fasd_fixed_step_whole_run_matches_reference(lat400):
    """GLU_GFIX_SD build: no line search, so the whole run agrees (slice 7
    also takes a continuation run past max_iters = 650)."""
    g = lat400
    d = _dims(g)
    r = gfix.coulomb_fix(g["links"], d, 0.09, ACC, 650, "FASD",
                         sd_fixed_step=True, traj_cap=d[3] * 2000)
    assert r.iters == int(g["coulomb_fasd_sd_iters"])
    assert r.slice_iters.max() > 650
    ref = _split(g["coulomb_fasd_sd_traj_theta"], r.slice_iters)
    got = _gpu_slices(r, d[3])
    for t in range(d[3]):
        assert len(got[t]) == r.slice_iters[t]
        # rounding-limited near theta ~ 1e-14: 5e-8 relative there is
        # ~1e-22 absolute, the derivative's FP64 rounding floor
        assert _rel(got[t], ref[t]).max() < 5e-8
    assert np.all(r.slice_theta < ACC)
    assert np.abs(r.links - g["coulomb_fasd_sd_links"]).max() < 1e-11


def test_facg_matches_reference_and_oracle(oracle, lat400):
    g = lat400
    d = _dims(g)
    r = gfix.coulomb_fix(g["links"], d, 0.09, ACC, 650, "FACG",
                         traj_cap=d[3] * 1000)
    o = oracle.coulomb(g["links"], d, 0.09, ACC, 650, "FACG", traj_cap=20000)
    assert abs(r.iters - int(g["coulomb_facg_iters"])) <= 8
    assert np.all(r.slice_theta < ACC)
    got = _gpu_slices(r, d[3])
    # the oracle's slice lengths split the reference's concatenation the
    # way the reference ran (its prefixes agree to 1e-10 for 23+ entries)
    ref = _split(g["coulomb_facg_traj_theta"], o["slice_iters"] + 1)
    orc = _split(o["traj_theta"], o["slice_iters"] + 1)
    for t in range(d[3]):
        # SD start + 11 CG steps of every slice
        assert _rel(got[t][:12], ref[t][:12]).max() < 1e-10
        assert _rel(got[t][:12], orc[t][:12]).max() < 1e-10
        assert abs(int(r.slice_iters[t]) - int(o["slice_iters"][t])) <= 4
    # the end points of different line-search paths agree to ~sqrt(theta)
    assert np.abs(r.links - g["coulomb_facg_links"]).max() < 1e-6


def test_facg_heatbath_config_matches_oracle(oracle, hb8):
    g = hb8
    d = _dims(g)
    r = gfix.coulomb_fix(g["links"], d, 0.08, ACC, 2000, "FACG",
                         traj_cap=d[3] * 1000)
    o = oracle.coulomb(g["links"], d, 0.08, ACC, 2000, "FACG", traj_cap=20000)
    assert np.all(r.slice_theta < ACC) and r.restarts == 0
    assert abs(r.iters - o["iters"]) <= 0.05 * o["iters"]
    got = _gpu_slices(r, d[3])
    orc = _split(o["traj_theta"], o["slice_iters"] + 1)
    for t in range(d[3]):
        assert _rel(got[t][:10], orc[t][:10]).max() < 1e-10
    # gauge invariance: plaquette unchanged
    _, _, p0 = gfix.observables(g["links"], d)
    _, _, p1 = gfix.observables(r.links, d)
    assert abs(p1 - p0) < 1e-13


def test_fasd_line_search_matches_oracle(oracle, lat400):
    g = lat400
    d = _dims(g)
    r = gfix.coulomb_fix(g["links"], d, 0.09, ACC, 650, "FASD",
                         traj_cap=d[3] * 2000)
    o = oracle.coulomb(g["links"], d, 0.09, ACC, 650, "FASD", traj_cap=20000)
    assert np.all(r.slice_theta < ACC)
    got = _gpu_slices(r, d[3])
    orc = _split(o["traj_theta"], o["slice_iters"])
    for t in range(d[3]):
        assert _rel(got[t][:20], orc[t][:20]).max() < 1e-10
    assert abs(r.iters - o["iters"]) <= 0.05 * o["iters"]


@pytest.mark.parametrize("dims", [(5, 5, 5, 4), (6, 4, 3, 5)])
def test_odd_extents_match_oracle(oracle, dims):
    """Odd and mixed-radix slices (generic FFT passes, all-site line search)."""
    U = _smooth_links(dims, 0.2, 11)
    r = gfix.coulomb_fix(U, dims, 0.08, ACC, 1000, "FACG", traj_cap=dims[3] * 1000)
    o = oracle.coulomb(U, dims, 0.08, ACC, 1000, "FACG", traj_cap=20000)
    assert np.all(r.slice_theta < ACC)
    got = _gpu_slices(r, dims[3])
    orc = _split(o["traj_theta"], o["slice_iters"] + 1)
    for t in range(dims[3]):
        n = min(10, len(orc[t]))
        assert _rel(got[t][:n], orc[t][:n]).max() < 1e-10
    assert abs(r.iters - o["iters"]) <= max(4, 0.05 * o["iters"])


def test_fixed_links_take_one_step_per_slice(lat400):
    """Already in Coulomb gauge: every slice stops after its first CG step
    (steep_step_FACG always takes one), so GLU returns Lt."""
    g = lat400
    d = _dims(g)
    r = gfix.coulomb_fix(g["coulomb_facg_links"], d, 0.09, 1e-12, 650, "FACG")
    assert r.iters == d[3]
    assert np.all(r.slice_iters == 1)


def test_device_entry_matches_host_entry(lat400):
    g = lat400
    d = _dims(g)
    h = gfix.coulomb_fix(g["links"], d, 0.09, ACC, 650, "FACG")
    dev = torch.from_numpy(np.ascontiguousarray(g["links"]).view(np.float64).copy()).cuda()
    r = gfix.coulomb_fix_device(dev.data_ptr(), d, 0.09, ACC, 650, "FACG")
    U = dev.cpu().numpy().view(np.complex128).reshape(h.links.shape)
    assert r.iters == h.iters
    assert np.abs(U - h.links).max() == 0.0


def test_glu_named_coulomb_reunitarises(lat400):
    g = lat400
    d = _dims(g)
    U, it = gfix.Coulomb(g["links"], d, 0.09, ACC, 650)
    assert abs(it - int(g["coulomb_facg_iters"])) <= 8
    M = U.reshape(-1, 3, 3)
    err = np.abs(M @ np.conj(np.swapaxes(M, -1, -2)) - np.eye(3)).max()
    assert err < 1e-14


@pytest.mark.parametrize("case", ["lat400", "hb8"])
def test_mixed_precision_reaches_fp64_accuracy(case, request):
    """FP32 phase to theta < 1e-9 per slice, FP64 polish to 1e-14: the same
    accuracy, the links on the same gauge orbit, and the FP64 fix's gauge."""
    g = request.getfixturevalue(case)
    d = _dims(g)
    alpha = 0.09 if case == "lat400" else 0.08
    r64 = gfix.coulomb_fix(g["links"], d, alpha, ACC, 2000, "FACG")
    r = gfix.coulomb_fix(g["links"], d, alpha, ACC, 2000, "FACG",
                         precision="MIXED", switch_theta=1e-9)
    assert np.all(r.slice_theta < ACC)
    assert 0 < r.iters_fp32 < r.iters
    assert np.all(r.slice_iters > 0)
    _, _, p0 = gfix.observables(g["links"], d)
    _, _, p1 = gfix.observables(r.links, d)
    assert abs(p1 - p0) < 1e-13
    # Coulomb gauge leaves one global SU(3) rotation per slice free, and the
    # FP32 rounding of the derivative's zero mode moves it (~1e-4 here); the
    # traces of the spatial links are blind to it and pin the local gauge to
    # the distance theta < 1e-14 leaves open
    # (a small Faddeev-Popov eigenvalue can stretch that to ~1e-6); the
    # spatial functional, second order at the solution, agrees to 1e-13
    tr = lambda U: np.trace(U[:, :3], axis1=-2, axis2=-1)  # noqa: E731
    assert np.abs(tr(r.links) - tr(r64.links)).max() < 1e-5
    fs = lambda U: 1.0 - tr(U).real.sum() / (9.0 * U.shape[0])  # noqa: E731
    assert abs(fs(r.links) - fs(r64.links)) < 1e-13


def test_mixed_precision_on_a_thermalised_configuration(monkeypatch):
    """A genuine beta 6.0 heatbath configuration (16^3x32, generated on the
    GPU): slices stuck on a theta plateau in FP32 hand over to FP64 by the
    per-slice stall rule; with it and without it every slice reaches
    theta < 1e-14 on the input's gauge orbit."""
    from glu_b200.workload import heatbath_config
    d = (16, 16, 16, 32)
    U = heatbath_config(d, seed=9, iterations=300)
    p0 = gfix.observables(U, d)[2]
    for stall in (None, "0"):
        if stall is None:
            monkeypatch.delenv("GLU_GFIX_STALL", raising=False)
        else:
            monkeypatch.setenv("GLU_GFIX_STALL", stall)
        r = gfix.coulomb_fix(U, d, 0.08, ACC, 20000, "FACG", precision="MIXED",
                             switch_theta=1e-9)
        assert np.all(r.slice_theta < ACC)
        assert 0 < r.iters_fp32 < r.iters
        assert abs(gfix.observables(r.links, d)[2] - p0) < 1e-12


@pytest.mark.parametrize("blocks", [[(0, 4), (4, 8)], [(0, 2), (2, 5), (5, 8)]])
def test_slice_blocks_equal_whole_lattice(lat400, blocks):
    """gfix_coulomb_slices on blocks of slices (one per rank in a sharded
    fix), the boundary fields passed along the ring, then
    gfix_coulomb_slices_finish: bit-equal to gfix_coulomb on the whole."""
    import ctypes as C
    from glu_b200 import _lib
    from glu_b200._lib import GfixResult, check
    g = lat400
    d = _dims(g)
    whole = gfix.coulomb_fix(g["links"], d, 0.09, ACC, 650, "FACG")
    lib = _lib.load()
    p, _, _ = gfix._params(0.09, ACC, 650, "FACG", False, "FP64", 1e-9, 0)
    lcu = d[0] * d[1] * d[2]
    U = np.ascontiguousarray(g["links"])
    dev, gf, gl, its = [], [], [], []
    for t0, t1 in blocks:
        blk = torch.from_numpy(U[t0 * lcu:t1 * lcu].view(np.float64).reshape(-1).copy()).cuda()
        dims = (C.c_size_t * 4)(d[0], d[1], d[2], t1 - t0)
        gfirst = torch.empty(9 * lcu * 2, dtype=torch.float64, device="cuda")
        glast = torch.empty_like(gfirst)
        r = GfixResult()
        th = np.zeros(t1 - t0)
        it = np.zeros(t1 - t0, dtype=np.uintp)
        check(lib.gfix_coulomb_slices(blk.data_ptr(), dims, C.byref(p), C.byref(r),
                                      th.ctypes.data_as(C.POINTER(C.c_double)),
                                      it.ctypes.data_as(C.POINTER(C.c_size_t)),
                                      gfirst.data_ptr(), glast.data_ptr()))
        dev.append((blk, dims))
        gf.append(gfirst)
        gl.append(glast)
        its.append(it.astype(np.int64))
    for k, (blk, dims) in enumerate(dev):
        check(lib.gfix_coulomb_slices_finish(blk.data_ptr(), dims, gl[k].data_ptr(),
                                             gf[(k + 1) % len(dev)].data_ptr()))
    got = np.concatenate([b.cpu().numpy() for b, _ in dev]).view(np.complex128)
    assert np.array_equal(got.reshape(whole.links.shape), whole.links)
    assert np.array_equal(np.concatenate(its), whole.slice_iters)
