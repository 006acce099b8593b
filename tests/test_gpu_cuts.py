"""Momentum-space gluon measurements on the GPU (gfix_cuts_*) against the
oracle and against GLU's own output files: the transverse / longitudinal
propagators (GLUON_PROPS), the MOMgg g2, g3 (EXCEPTIONAL) and the fields
(FIELDS) for every momentum cut, on compile-time and generic FFT extents."""
import json
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import cuts, gfix  # noqa: E402
from glu_b200.workload import random_su3  # noqa: E402
from oracle import cuts_oracle as CO  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden" / "cuts"
CASES = json.loads((GOLD / "cases.json").read_text())
OUT_KEYS = {"GLUON_PROPS": ("transverse", "longitudinal"),
            "EXCEPTIONAL": ("g2", "g3"), "FIELDS": ("fields", None)}
TOL = 1e-12  # relative to the largest |value| of the first output


def _links(dims, seed=5):
    rng = np.random.default_rng(seed)
    V = int(np.prod(dims))
    return random_su3(V * 4, rng).reshape(V, 4, 3, 3)


def _close(a, b, scale):
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= TOL * scale


@pytest.mark.parametrize("case", CASES, ids=[c["file"] for c in CASES])
def test_files_match_glu(lat400, tmp_path, case):
    """cuts_struct's file: GLU's name, momentum list bit for bit, values to
    rounding."""
    dims = tuple(int(d) for d in lat400["dims"])
    info = cuts.CutInfo(case["cuttype"], case["mom_cut"], case["field_definition"],
                        case["maxmom"], case["angle"], case["cyl_width"])
    path, _ = cuts.cuts_struct(lat400[case["links"]], dims, info,
                               where=str(tmp_path) + "/", flow=case["flow"])
    assert path.name == case["file"]
    got = cuts.read_output(path, case["cuttype"])
    ref = cuts.read_output(GOLD / case["file"], case["cuttype"])
    assert np.array_equal(got["mom"], ref["mom"])
    for k in OUT_KEYS[case["cuttype"]]:
        if k:
            assert _close(got[k], ref[k], np.abs(ref[OUT_KEYS[case["cuttype"]][0]]).max())


DIMS = [(8, 8, 8, 8),     # compile-time xy and zt passes
        (8, 8, 8, 16),    # compile-time, zt tile of 4 columns
        (4, 4, 4, 8),     # generic passes
        (6, 6, 6, 12),    # generic, radix 3
        (10, 10, 10, 10)]  # generic, radix 5
CUTS = [("SPHERICAL_CUT", 12, 0, 1.0), ("HYPERCUBIC_CUT", 3, 0, 1.0),
        ("CYLINDER_CUT", 20, 0, 1.0), ("CONICAL_CUT", 20, 40, 1.5)]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("cuttype", ["GLUON_PROPS", "EXCEPTIONAL", "FIELDS"])
@pytest.mark.parametrize("definition", ["LINEAR", "LOGARITHMIC"])
def test_measure_matches_oracle(dims, cuttype, definition):
    U = _links(dims)
    for mc, mm, ang, w in CUTS:
        info = cuts.CutInfo(cuttype, mc, definition, mm, ang, w)
        r = cuts.measure(U, dims, info)
        o = CO.measure(U, dims, cuts.CUTTYPES[cuttype], cuts.MOM_CUTS[mc], mm, ang, w,
                       cuts.FIELD_DEFINITIONS[definition])
        assert np.array_equal(r["mom"], o["mom"])
        k0, k1 = OUT_KEYS[cuttype]
        scale = np.abs(o["out0"]).max()
        assert _close(r[k0], o["out0"], scale), (mc, k0)
        if k1:
            assert _close(r[k1], o["out1"], scale), (mc, k1)
        assert abs(r["pspace_err"] - o["pspace_err"]) <= 1e-12 * o["pspace_err"]


def test_log_of_identity_and_near_identity_links():
    """The logarithm's near-identity eigenvalue branch, and exact identity
    links (log 0; GLU's routine leaves its output unwritten there)."""
    from scipy.linalg import expm
    dims = (8, 8, 8, 8)
    V = int(np.prod(dims))
    U = _links(dims, 13)
    rng = np.random.default_rng(4)
    sel = rng.choice(V * 4, V // 2, replace=False)
    flat = U.reshape(V * 4, 3, 3)
    for k, i in enumerate(sel):
        if k % 4 == 0:
            flat[i] = np.eye(3)
        else:
            a = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
            h = (a + a.conj().T) / 2
            h -= np.trace(h) / 3 * np.eye(3)
            flat[i] = expm(1j * 3e-7 * h)
    info = cuts.CutInfo("FIELDS", "SPHERICAL_CUT", "LOGARITHMIC", 6)
    r = cuts.measure(U, dims, info)
    o = CO.measure(U, dims, 2, 1, 6, 0, 1.0, 1)
    assert _close(r["fields"], o["out0"], np.abs(o["out0"]).max())


def test_device_entry_matches_host_entry():
    dims = (8, 8, 8, 16)
    U = _links(dims, 9)
    info = cuts.CutInfo("GLUON_PROPS", "CYLINDER_CUT", "LINEAR", 30, 0, 1.0)
    r = cuts.measure(U, dims, info)
    d = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).cuda()
    rd = cuts.measure_device(d, dims, info)
    assert np.array_equal(r["transverse"], rd["transverse"])
    assert np.array_equal(r["longitudinal"], rd["longitudinal"])


def test_landau_fixed_fields_are_transverse():
    """After a Landau fix to theta < 1e-14 the longitudinal propagator
    vanishes to theta's level while the transverse one stays O(1): the
    transform, the half-step phase and the projector agree with the lattice
    Landau condition at any size."""
    from glu_b200.workload import tiled_config
    dims = (16, 16, 16, 32)
    U = tiled_config(dims, seed=3)  # the shipped 4^3x8 field, tiled and rotated
    res = gfix.landau_fix(U, dims, accuracy=1e-14, traj_cap=0)
    info = cuts.CutInfo("GLUON_PROPS", "SPHERICAL_CUT", "LINEAR", 40, 0, 1.0)
    r = cuts.measure(res.links, dims, info)
    assert np.abs(r["transverse"]).max() > 1e-3
    assert np.abs(r["longitudinal"]).max() < 1e-10 * np.abs(r["transverse"]).max()


def test_bad_arguments_raise():
    U = _links((4, 4, 4, 8))
    with pytest.raises(cuts.CutsError):
        cuts.measure(U, (4, 4, 4, 8), cuts.CutInfo(cuttype="STATIC_POTENTIAL"))
    with pytest.raises(cuts.CutsError):
        cuts.measure(_links((4, 4, 4, 11)), (4, 4, 4, 11), cuts.CutInfo())  # prime 11
