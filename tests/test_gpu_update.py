"""Configuration generation on the GPU (gfix_heatbath, gfix_overrelax)
against GLU: the over-relaxation value for value (GLU's OR_lattice on the
same links, committed in lat400.npz), the heatbath in distribution (GLU's
average plaquette at beta 6.0 and 5.7, tests/golden/heatbath_glu.json),
plus unitarity, reproducibility and continuation."""
import json
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import gfix, update  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden"


def _dims(g):
    return tuple(int(d) for d in g["dims"])


def test_overrelax_matches_glu(lat400):
    U = update.overrelax(lat400["links"], _dims(lat400), 2)
    ref = lat400["or2_links"]
    assert np.abs(U - ref).max() < 1e-12


def test_overrelax_matches_glu_on_heatbath_config(reference, hb8):
    dims = _dims(hb8)
    reference.setup(dims)
    reference.put_links(hb8["links"])
    reference.overrelax(3)
    U = update.overrelax(hb8["links"], dims, 3)
    assert np.abs(U - reference.get_links()).max() < 1e-11


def test_overrelax_keeps_the_action(hb8):
    dims = _dims(hb8)
    p0 = gfix.av_plaquette(hb8["links"], dims)
    U = update.overrelax(hb8["links"], dims, 5)
    assert abs(gfix.av_plaquette(U, dims) - p0) < 1e-13
    assert np.abs(U - hb8["links"]).max() > 0.1  # the links did move


def _binned(x, b):
    n = len(x) // b
    m = np.asarray(x[: n * b]).reshape(n, b).mean(axis=1)
    return m.mean(), m.std(ddof=1) / np.sqrt(n)


@pytest.mark.parametrize("run", json.loads((GOLD / "heatbath_glu.json").read_text())["runs"],
                         ids=lambda r: "beta%.1f" % r["beta"])
def test_heatbath_plaquette_matches_glu(run):
    dims = (8, 8, 8, 8)
    _, p = update.heatbath(update.unit_config(dims), dims, run["beta"],
                           run["therm"] + run["iterations"], run["n_or"], seed=2024)
    mean, err = _binned(p[run["therm"]:], run["bin"])
    sigma = np.hypot(err, run["err"])
    assert abs(mean - run["mean"]) < 5 * sigma, (mean, err, run["mean"], run["err"])


def test_links_stay_in_su3():
    dims = (8, 8, 8, 16)
    U, _ = update.heatbath(update.unit_config(dims), dims, 5.9, 20, 2, seed=3)
    eye = np.eye(3)
    assert np.abs(U @ np.conj(np.swapaxes(U, -1, -2)) - eye).max() < 1e-13
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-13


def test_reproducible_and_continuable():
    dims = (8, 8, 8, 8)
    U0 = update.unit_config(dims)
    a, pa = update.heatbath(U0, dims, 6.0, 10, 1, seed=99)
    b, _ = update.heatbath(U0, dims, 6.0, 6, 1, seed=99)
    b, pb = update.heatbath(b, dims, 6.0, 4, 1, seed=99, first_iteration=6)
    assert np.array_equal(a, b)
    assert pa[-1] == pb[-1]
    c, _ = update.heatbath(U0, dims, 6.0, 10, 1, seed=100)
    assert not np.array_equal(a, c)


def test_device_entry_matches_host_entry():
    dims = (8, 8, 8, 8)
    U0 = update.unit_config(dims)
    a, pa = update.heatbath(U0, dims, 5.8, 5, 2, seed=5)
    d = torch.from_numpy(U0.view(np.float64).reshape(-1).copy()).cuda()
    pd = update.heatbath_device(d, dims, 5.8, 5, 2, seed=5)
    assert np.array_equal(d.cpu().numpy().view(np.complex128).reshape(a.shape), a)
    assert np.array_equal(pa, pd)


def test_odd_extents_are_rejected():
    with pytest.raises(update.UpdateError):
        update.heatbath(update.unit_config((4, 4, 4, 5)), (4, 4, 4, 5), 6.0, 1)
