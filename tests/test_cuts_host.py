"""Momentum-space gluon measurements, host side: the oracle
(oracle/cuts_oracle.py) pinned against GLU's own cuts_struct -- through the
committed output files of tests/golden/cuts/ (written by GLU) and, where the
reference build is present, against fresh GLU runs -- and the library's
momentum list (gfix_cut_veclist, host code) against GLU's compute_veclist,
bit for bit."""
import json
from pathlib import Path

import numpy as np
import pytest

from glu_b200 import cuts
from oracle import cuts_oracle as CO

GOLD = Path(__file__).resolve().parent / "golden" / "cuts"
CASES = json.loads((GOLD / "cases.json").read_text())
OUT_KEYS = {"GLUON_PROPS": ("transverse", "longitudinal"),
            "EXCEPTIONAL": ("g2", "g3"), "FIELDS": ("fields", None)}


def _oracle(links, dims, case):
    return CO.measure(links, dims, cuts.CUTTYPES[case["cuttype"]],
                      cuts.MOM_CUTS[case["mom_cut"]], case["maxmom"],
                      case["angle"], case["cyl_width"],
                      cuts.FIELD_DEFINITIONS[case.get("field_definition", "LINEAR")])


@pytest.mark.parametrize("case", CASES, ids=[c["file"] for c in CASES])
def test_oracle_matches_glu_output_files(lat400, case):
    dims = tuple(int(d) for d in lat400["dims"])
    ref = cuts.read_output(GOLD / case["file"], case["cuttype"])
    o = _oracle(lat400[case["links"]], dims, case)
    assert np.array_equal(ref["mom"], o["mom"])
    k0, k1 = OUT_KEYS[case["cuttype"]]
    a = ref[k0]
    b = o["out0"]
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    if k1:
        assert np.abs(ref[k1] - o["out1"]).max() <= 1e-13 * np.abs(ref[k0]).max()


def _random_links(dims, seed):
    from glu_b200.workload import random_su3
    rng = np.random.default_rng(seed)
    V = int(np.prod(dims))
    return random_su3(V * 4, rng).reshape(V, 4, 3, 3)


@pytest.mark.parametrize("dims", [(4, 4, 4, 8), (6, 6, 6, 12), (8, 8, 8, 8)])
@pytest.mark.parametrize("cuttype", ["GLUON_PROPS", "EXCEPTIONAL", "FIELDS"])
@pytest.mark.parametrize("definition", ["LINEAR", "LOGARITHMIC"])
def test_oracle_matches_glu_runs(reference, dims, cuttype, definition):
    U = _random_links(dims, 11)
    case = dict(cuttype=cuttype, mom_cut="CONICAL_CUT", maxmom=12, angle=45,
                cyl_width=1.5, field_definition=definition)
    reference.setup(dims)
    reference.put_links(U)
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        p = reference.cuts(td, cuts.CUTTYPES[cuttype], 3, 12,
                           cuts.FIELD_DEFINITIONS[definition], 45, 1.5, flow=3)
        ref = cuts.read_output(p, cuttype)
    o = _oracle(U, dims, case)
    assert np.array_equal(ref["mom"], o["mom"])
    k0, k1 = OUT_KEYS[cuttype]
    assert np.abs(ref[k0] - o["out0"]).max() <= 1e-12 * np.abs(ref[k0]).max()
    if k1:
        assert np.abs(ref[k1] - o["out1"]).max() <= 1e-12 * np.abs(ref[k0]).max()


VEC_DIMS = [(4, 4, 4, 8), (6, 6, 6, 12), (8, 8, 8, 8), (8, 8, 8, 16), (12, 12, 12, 24),
            (16, 16, 16, 32)]
VEC_CUTS = [("HYPERCUBIC_CUT", 3, 0, 1.0), ("SPHERICAL_CUT", 20, 0, 1.0),
            ("CYLINDER_CUT", 40, 0, 1.0), ("CYLINDER_CUT", 64, 0, 0.5),
            ("CONICAL_CUT", 40, 30, 2.0), ("CONICAL_CUT", 100, 70, 1.0)]


@pytest.mark.parametrize("dims", VEC_DIMS)
@pytest.mark.parametrize("cut", VEC_CUTS, ids=lambda c: f"{c[0]}-{c[1]}")
def test_library_veclist_equals_glu(reference, dims, cut):
    mc, mm, ang, w = cut
    reference.setup(dims)
    ref, ref_idx = reference.veclist(6, cuts.MOM_CUTS[mc], mm, ang, w)
    got = cuts.veclist(dims, cuts.CutInfo("GLUON_PROPS", mc, "LINEAR", mm, ang, w))
    assert len(ref) > 0
    assert np.array_equal(got, ref)


def test_library_veclist_of_the_fixture_cases(lat400):
    dims = tuple(int(d) for d in lat400["dims"])
    for case in CASES:
        ref = cuts.read_output(GOLD / case["file"], case["cuttype"])
        info = cuts.CutInfo(case["cuttype"], case["mom_cut"], "LINEAR", case["maxmom"],
                            case["angle"], case["cyl_width"])
        assert np.array_equal(cuts.veclist(dims, info), ref["mom"])


def test_unsupported_modes_raise():
    with pytest.raises(cuts.CutsError):
        cuts.CutInfo("NON_EXCEPTIONAL").c()


def _near_identity(V, eps, rng):
    """links exp(i eps H) with H random traceless Hermitian"""
    from scipy.linalg import expm
    out = np.empty((V, 3, 3), dtype=np.complex128)
    for i in range(V):
        a = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        h = (a + a.conj().T) / 2
        h -= np.trace(h) / 3 * np.eye(3)
        out[i] = expm(1j * eps * h)
    return out


def test_oracle_log_near_identity_matches_glu(reference):
    """GLU's near-identity eigenvalue branch (1 - Re tr U / 3 < 1e-12)."""
    dims = (4, 4, 4, 4)
    V = 256
    rng = np.random.default_rng(5)
    U = _near_identity(V * 4, 3e-7, rng).reshape(V, 4, 3, 3)
    assert (1.0 - np.trace(U, axis1=-2, axis2=-1).real / 3.0 < 1e-12).mean() > 0.5
    reference.setup(dims)
    reference.put_links(U)
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        p = reference.cuts(td, 2, 1, 3, 1, 0, 1.0, flow=1)
        ref = cuts.read_output(p, "FIELDS")
    o = CO.measure(U, dims, 2, 1, 3, 0, 1.0, definition=1)
    assert np.abs(ref["fields"] - o["out0"]).max() <= 1e-10 * np.abs(ref["fields"]).max()
