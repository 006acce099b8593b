"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run from the repository root after ``make -C oracle``:

    python tests/golden/make_golden.py

It needs the reference sources (for the shipped 4^3x8 configuration and the
reference build in oracle/_ref).  Outputs are committed, so the tests (and the
GPU box, which has no reference tree) only read them.

Fixtures
--------
lat400.npz   4^3x8 configuration shipped with the reference (CONF/lat..400),
             read by GLU's own NERSC reader, plus reference results:
               Landau FACG / FASD (line-search SD) / FASD (GLU_GFIX_SD build,
               fixed step), Coulomb FACG / FASD (GLU_GFIX_SD build)
cuts/        GLU's momentum-space output files (G2F2 / MOMgg / MATS) of the
             Landau-fixed lat400 links, with cases.json
heatbath_glu.json  GLU's heatbath + over-relaxation plaquette statistics
             (8^4, unit start) at beta 6.0 and 5.7; lat400.npz["or2_links"]
             holds the fixture links after two of GLU's over-relaxation sweeps
hb8.npz      8^4 SU(3) configuration from GLU's heatbath (beta 6.0, cold
             start, seed 1, 500 sweeps of KP heatbath + 4 over-relaxation,
             8 OpenMP threads), plus reference Landau FACG (alpha 0.08,
             theta < 1e-14)

Each solve stores the 1-thread reference trajectory (theta and functional at
every derivative evaluation, SD start included), the iteration count, the
final theta and the final links (hb8: every 8th site), and -- for Landau
FACG -- the first 60
in-loop thetas of the same reference run with 8 OpenMP threads.  The two
reference runs differ only in summation order; their distance is the
reference's own reproducibility envelope used as the trajectory tolerance.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import REF_BIN, Reference  # noqa: E402

# the reference's source tree: an overridable default (GLU_REFERENCE)
REF = Path(os.environ.get("GLU_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent
ENVELOPE_ITERS = 60

HB_INPUT = """MODE = HEATBATH
HEADER = UNIT
    DIM_0 = 8
    DIM_1 = 8
    DIM_2 = 8
    DIM_3 = 8
CONFNO = 0
RANDOM_TRANSFORM = NO
SEED = 1
GFTYPE = LANDAU
    GF_TUNE = 0.08
    ACCURACY = 14
    MAX_ITERS = 650
CUTTYPE = GLUON_PROPS
    FIELD_DEFINITION = LINEAR
    MOM_CUT = CYLINDER_CUT
    MAX_T = 7
    MAXMOM = 4
    CYL_WIDTH = 2.0
    ANGLE = 60
    OUTPUT = ./
SMEARTYPE = APE
    DIRECTION = ALL
    SMITERS = 100
    ALPHA1 = 0.6
    ALPHA2 = 0.4
    ALPHA3 = 0.2
U1_MEAS = U1_RECTANGLE
    U1_ALPHA = 0.07957753876221914
    U1_CHARGE = -1.0
CONFIG_INFO = glu_b200_golden
    STORAGE = NERSC_GAUGE
BETA = 6.0
    ITERS = 501
    MEASURE = 100
    OVER_ITERS = 4
    SAVE = 500
    THERM = 0
"""


def heatbath_8x4(tmp: Path) -> Path:
    (tmp / "in_hb").write_text(HB_INPUT)
    env = dict(os.environ, OMP_NUM_THREADS="8")
    subprocess.run([str(REF_BIN), "-i", "in_hb", "-c", "hb8"], cwd=tmp,
                   env=env, check=True, stdout=subprocess.DEVNULL)
    return tmp / "hb8.500"


def envelope(R: Reference, links, alpha: float, max_k: int) -> np.ndarray:
    """In-loop theta after k = 1..max_k FACG iterations with 8 threads.

    acc = 1e-30 never converges and never triggers a continuation run, so
    FACG stops after exactly k iterations and returns that iteration's theta.
    """
    R.set_threads(8)
    out = []
    for k in range(1, max_k + 1):
        R.put_links(links)
        R.set_alpha(alpha)
        out.append(R.landau_fa(1e-30, k, "FACG")["theta"])
    R.set_threads(1)
    return np.array(out)


def landau_case(R: Reference, links, alpha, algo, acc=1e-14, max_iters=650):
    R.put_links(links)
    R.set_alpha(alpha)
    r = R.landau_fa(acc, max_iters, algo, traj_cap=100000)
    r["links"] = R.get_links()
    return r


def coulomb_case(R: Reference, links, alpha, algo, acc=1e-14, max_iters=650):
    R.put_links(links)
    R.set_alpha(alpha)
    r = R.coulomb_fa(acc, max_iters, algo, traj_cap=100000)
    r["links"] = R.get_links()
    return r


def pack(prefix: str, r: dict, store: dict, links=True):
    store[f"{prefix}_iters"] = np.int64(r["iters"])
    if "theta" in r:
        store[f"{prefix}_theta"] = np.float64(r["theta"])
    store[f"{prefix}_traj_theta"] = r["traj_theta"]
    if "traj_func" in r:
        store[f"{prefix}_traj_func"] = r["traj_func"]
    if links:
        store[f"{prefix}_links"] = r["links"]


DIAG_KEYS = ("splink", "tlink", "all", "link", "link_max_trace", "const_lin",
             "const_log")


def diagnostics(R: Reference, links) -> np.ndarray:
    """GLU's all_links, indivlinks and const_time of `links` (the lattice
    set up in R): the 7 values of Reference.diagnostics."""
    R.put_links(links)
    return np.array(R.diagnostics())


def add_diagnostics() -> None:
    """Adds GLU's link diagnostics of the input and of the fixed links to
    the existing fixtures (lat400: input, Landau FACG, Coulomb FACG links)."""
    R = Reference()
    g = dict(np.load(OUT / "lat400.npz"))
    R.setup(tuple(int(d) for d in g["dims"]), 1, 0.08)
    for key, links in (("input", g["links"]), ("landau", g["landau_facg_links"]),
                       ("coulomb", g["coulomb_facg_links"])):
        g[f"diag_{key}"] = diagnostics(R, links)
    np.savez(OUT / "lat400.npz", **g)
    print("lat400 diagnostics:", {k: v for k, v in g.items() if k.startswith("diag")})


def nersc_fixture() -> None:
    """tests/golden/lat400.nersc: the 4^3x8 fixture links as a NERSC file
    (4D_SU3_GAUGE, IEEE64BIG), written by this numpy encoder and checked by
    GLU's own reader (checksum, plaquette and link trace of the header, and
    every link read back equal to the fixture's)."""
    g = dict(np.load(OUT / "lat400.npz"))
    U = g["links"]
    dims = tuple(int(d) for d in g["dims"])
    top = np.ascontiguousarray(U[:, :, :2, :]).view(np.float64)
    ck = int(np.frombuffer(top.astype("<f8").tobytes(), "<u4").sum(dtype=np.uint64)
             & 0xFFFFFFFF)
    trace = float(np.trace(U, axis1=-2, axis2=-1).real.mean() / 3.0)
    hdr = ["BEGIN_HEADER", "HDR_VERSION = 1.0", "DATATYPE = 4D_SU3_GAUGE",
           "STORAGE_FORMAT = 1.0"]
    hdr += [f"DIMENSION_{k + 1} = {dims[k]}" for k in range(4)]
    hdr += ["LINK_TRACE = %1.15f" % trace, "PLAQUETTE = %1.15f" % float(g["plaquette"])]
    hdr += [f"BOUNDARY_{k + 1} = PERIODIC" for k in range(4)]
    hdr += ["CHECKSUM = %x" % ck, "ENSEMBLE_ID = glu_b200_fixture",
            "SEQUENCE_NUMBER = 400", "FLOATING_POINT = IEEE64BIG", "END_HEADER"]
    path = OUT / "lat400.nersc"
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode("ascii"))
        f.write(top.astype(">f8").tobytes())
    R = Reference()
    back = R.read_file(path)
    assert np.array_equal(back, U), "GLU read the file differently"
    print("lat400.nersc: checksum %x accepted by GLU's reader" % ck)


def ildg_fixture() -> None:
    """tests/golden/lat400.ildg: the 4^3x8 fixture links written by GLU's own
    ILDG writer (which reunitarises them first); the links GLU reads back
    are stored as lat400.npz["ildg_links"]."""
    g = dict(np.load(OUT / "lat400.npz"))
    R = Reference()
    R.setup(tuple(int(d) for d in g["dims"]), 1, 0.08)
    R.put_links(g["links"])
    path = OUT / "lat400.ildg"
    path.unlink(missing_ok=True)  # GLU's writer does not overwrite
    R.write(path, "ILDG", "glu_b200 fixture")
    g["ildg_links"] = Reference().read_file(path, ildg=True)
    np.savez(OUT / "lat400.npz", **g)
    print("lat400.ildg written by GLU,", path.stat().st_size, "bytes")


# momentum-space cuts of the Landau-fixed 4^3x8 links written by GLU's
# cuts_struct: (CUTTYPE, MOM_CUT, MAXMOM, ANGLE, CYL_WIDTH, FIELD_DEFINITION)
CUT_CASES = [("GLUON_PROPS", "SPHERICAL_CUT", 6, 0, 1.0, "LINEAR"),
             ("GLUON_PROPS", "HYPERCUBIC_CUT", 2, 0, 1.0, "LINEAR"),
             ("GLUON_PROPS", "CYLINDER_CUT", 8, 0, 0.75, "LINEAR"),
             ("GLUON_PROPS", "CONICAL_CUT", 8, 40, 1.0, "LINEAR"),
             ("EXCEPTIONAL", "SPHERICAL_CUT", 6, 0, 1.0, "LINEAR"),
             ("FIELDS", "SPHERICAL_CUT", 2, 0, 1.0, "LINEAR"),
             ("GLUON_PROPS", "SPHERICAL_CUT", 6, 0, 1.0, "LOGARITHMIC"),
             ("EXCEPTIONAL", "CONICAL_CUT", 8, 40, 1.0, "LOGARITHMIC")]
CUT_DIRS = {"EXCEPTIONAL": 0, "FIELDS": 2, "GLUON_PROPS": 6}
CUT_TYPES = {"HYPERCUBIC_CUT": 0, "SPHERICAL_CUT": 1, "CYLINDER_CUT": 2,
             "CONICAL_CUT": 3}


def cuts_fixture() -> None:
    """tests/golden/cuts/: GLU's output files of its momentum-space
    measurements (src/Cuts/cuts.c) on lat400.npz["landau_facg_links"],
    configuration number 400, and cases.json naming their parameters."""
    import json
    g = dict(np.load(OUT / "lat400.npz"))
    dims = tuple(int(d) for d in g["dims"])
    out = OUT / "cuts"
    out.mkdir(exist_ok=True)
    R = Reference()
    cases = []
    for ct, mc, mm, ang, w, fd in CUT_CASES:
        R.setup(dims, 1, 0.08)
        R.put_links(g["landau_facg_links"])
        path = R.cuts(out, CUT_DIRS[ct], CUT_TYPES[mc], mm,
                      1 if fd == "LOGARITHMIC" else 0, ang, w, flow=400)
        cases.append(dict(file=path.name, cuttype=ct, mom_cut=mc, maxmom=mm,
                          angle=ang, cyl_width=w, field_definition=fd, flow=400,
                          links="landau_facg_links"))
        print(path.name, path.stat().st_size, "bytes")
    (out / "cases.json").write_text(json.dumps(cases, indent=1) + "\n")


# GLU's heatbath statistics (hb_update's update_lattice): 8^4 from the unit
# configuration, (beta, OR sweeps per heatbath, thermalisation, measured)
HB_RUNS = [(6.0, 4, 100, 1000), (5.7, 4, 100, 600)]
HB_BIN = 20


def binned(x, b):
    """mean and its error from bins of b consecutive measurements"""
    n = len(x) // b
    m = np.asarray(x[: n * b]).reshape(n, b).mean(axis=1)
    return float(m.mean()), float(m.std(ddof=1) / np.sqrt(n))


def update_fixture() -> None:
    """lat400.npz["or2_links"]: the fixture links after two of GLU's
    over-relaxation sweeps; tests/golden/heatbath_glu.json: GLU's average
    plaquette (binned mean and error) at each HB_RUNS point."""
    import json
    g = dict(np.load(OUT / "lat400.npz"))
    dims = tuple(int(d) for d in g["dims"])
    R = Reference()
    R.setup(dims, 1, 0.08)
    R.put_links(g["links"])
    R.overrelax(2)
    g["or2_links"] = R.get_links()
    np.savez(OUT / "lat400.npz", **g)
    runs = []
    d8 = (8, 8, 8, 8)
    unit = np.zeros((8 ** 4, 4, 3, 3), dtype=np.complex128)
    for k in range(3):
        unit[..., k, k] = 1.0
    for beta, n_or, therm, iters in HB_RUNS:
        R.setup(d8, 1, 0.08, 11)
        R.put_links(unit)
        p = R.heatbath(beta, therm + iters, n_or)
        mean, err = binned(p[therm:], HB_BIN)
        runs.append(dict(beta=beta, n_or=n_or, therm=therm, iterations=iters,
                         bin=HB_BIN, mean=mean, err=err))
        print("GLU heatbath beta %.2f: <P> = %.6f +- %.6f" % (beta, mean, err))
    (OUT / "heatbath_glu.json").write_text(
        json.dumps(dict(dims=list(d8), start="unit", runs=runs), indent=1) + "\n")


def main() -> None:
    if "--update" in sys.argv:
        update_fixture()
        return
    if "--cuts" in sys.argv:
        cuts_fixture()
        return
    if "--ildg" in sys.argv:
        ildg_fixture()
        return
    if "--diagnostics" in sys.argv:
        add_diagnostics()
        return
    if "--nersc" in sys.argv:
        nersc_fixture()
        return
    R = Reference()
    RSD = Reference(sd_build=True)

    # ---- 4^3 x 8 shipped configuration ---------------------------------
    cfg = REF / "CONF" / "lat..400"
    U = R.read_file(cfg)
    RSD.read_file(cfg)
    dims = np.array(R.dims, dtype=np.int64)
    st = dict(dims=dims, links=U, plaquette=np.float64(R.plaquette()),
              theta_test=np.float64(R.theta_test_lin()),
              functional=np.float64(R.gauge_functional()))
    pack("landau_facg", landau_case(R, U, 0.08, "FACG"), st)
    st["landau_facg_env8"] = envelope(R, U, 0.08, ENVELOPE_ITERS)
    pack("landau_fasd_ls", landau_case(R, U, 0.08, "FASD"), st)
    pack("landau_fasd_sd", landau_case(RSD, U, 0.08, "FASD"), st)
    pack("coulomb_facg", coulomb_case(R, U, 0.09, "FACG"), st)
    pack("coulomb_fasd_sd", coulomb_case(RSD, U, 0.09, "FASD"), st)
    np.savez(OUT / "lat400.npz", **st)
    print("lat400:", {k: v for k, v in st.items() if k.endswith("iters")})
    add_diagnostics()
    nersc_fixture()
    ildg_fixture()
    cuts_fixture()
    update_fixture()

    # ---- 8^4 heatbath configuration -------------------------------------
    with tempfile.TemporaryDirectory() as td:
        path = heatbath_8x4(Path(td))
        U = R.read_file(path)
        dims = np.array(R.dims, dtype=np.int64)
        st = dict(dims=dims, links=U, plaquette=np.float64(R.plaquette()),
                  theta_test=np.float64(R.theta_test_lin()),
                  functional=np.float64(R.gauge_functional()))
        r = landau_case(R, U, 0.08, "FACG")
        pack("landau_facg", r, st, links=False)
        # final links on every 8th site keep the fixture small
        st["sub_stride"] = np.int64(8)
        st["landau_facg_links_sub"] = r["links"][::8].copy()
        st["landau_facg_env8"] = envelope(R, U, 0.08, ENVELOPE_ITERS)
        np.savez(OUT / "hb8.npz", **st)
        print("hb8:", st["landau_facg_iters"], "plaquette", st["plaquette"])


if __name__ == "__main__":
    main()
