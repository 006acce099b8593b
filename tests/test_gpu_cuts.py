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


class _Site(__import__("ctypes").Structure):
    """GLU's struct site (src/Headers/GLU_types.h:269-273)"""
    import ctypes as C
    _fields_ = [("O", C.POINTER(C.POINTER(C.c_double))),
                ("neighbor", C.c_size_t * 4), ("back", C.c_size_t * 4)]


class _Latt(__import__("ctypes").Structure):
    """GLU's struct latt_info (src/Headers/GLU_types.h:229-243)"""
    import ctypes as C
    _fields_ = [("dims", C.c_size_t * 4), ("Lsq", C.c_size_t), ("Lcu", C.c_size_t),
                ("Volume", C.c_size_t), ("flow", C.c_size_t), ("gf_alpha", C.c_double),
                ("sm_alpha", C.c_double * 3), ("head", C.c_int), ("Seed", C.c_uint32 * 1),
                ("twiddles", C.c_double * 4), ("Nthreads", C.c_uint32),
                ("su2_data", C.c_void_p), ("argc", C.c_int)]


class _CutInfo(__import__("ctypes").Structure):
    """GLU's struct cut_info (src/Headers/GLU_types.h:94-103)"""
    import ctypes as C
    _fields_ = [("dir", C.c_int), ("type", C.c_int), ("max_mom", C.c_size_t),
                ("max_t", C.c_size_t), ("where", C.c_char * 256), ("definition", C.c_int),
                ("angle", C.c_size_t), ("cyl_width", C.c_double)]


def test_glu_named_cuts_struct_writes_glus_file(lat400, tmp_path, monkeypatch):
    """cuts_struct called as GLU calls it: a struct site lattice, Latt set,
    the file written into the working directory."""
    import ctypes as C
    from glu_b200 import _lib
    lib = _lib.load()
    case = next(c for c in CASES if c["cuttype"] == "GLUON_PROPS"
                and c["field_definition"] == "LOGARITHMIC")
    dims = tuple(int(d) for d in lat400["dims"])
    V = int(np.prod(dims))
    U = np.ascontiguousarray(lat400[case["links"]])
    rows = [(C.c_double * 18).from_buffer(U[i, mu]) for i in range(V) for mu in range(4)]
    ptrs = [(C.POINTER(C.c_double) * 4)(*[C.cast(rows[i * 4 + mu], C.POINTER(C.c_double))
                                          for mu in range(4)]) for i in range(V)]
    sites = (_Site * V)()
    for i in range(V):
        sites[i].O = C.cast(ptrs[i], C.POINTER(C.POINTER(C.c_double)))
    latt = _Latt.in_dll(lib, "Latt")
    for mu in range(4):
        latt.dims[mu] = dims[mu]
    latt.Volume = V
    latt.flow = case["flow"]
    ci = _CutInfo(cuts.CUTTYPES[case["cuttype"]], cuts.MOM_CUTS[case["mom_cut"]],
                  case["maxmom"], 0, b"./", 1, case["angle"], case["cyl_width"])
    lib.cuts_struct.restype = C.c_int
    lib.cuts_struct.argtypes = [C.POINTER(_Site), _CutInfo]
    monkeypatch.chdir(tmp_path)
    before = U.copy()
    assert lib.cuts_struct(sites, ci) == 0
    assert np.array_equal(U, before)  # the lattice is left as it was
    got = cuts.read_output(tmp_path / case["file"], "GLUON_PROPS")
    ref = cuts.read_output(GOLD / case["file"], "GLUON_PROPS")
    assert np.array_equal(got["mom"], ref["mom"])
    assert _close(got["transverse"], ref["transverse"], np.abs(ref["transverse"]).max())
    assert _close(got["longitudinal"], ref["longitudinal"], np.abs(ref["transverse"]).max())
    ci.dir = 1  # NON_EXCEPTIONAL: not provided
    assert lib.cuts_struct(sites, ci) == -1
