"""NERSC payload codec on the GPU (gfix_nersc_decode / _encode) against
GLU's reader: tests/golden/lat400.nersc was checked by GLU's own reader to
decode to the fixture links bit for bit (tests/golden/make_golden.py)."""
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from glu_b200 import nersc  # noqa: E402

FILE = Path(__file__).resolve().parent / "golden" / "lat400.nersc"


def test_read_matches_glu(lat400):
    U, dims, hdr = nersc.read(FILE)  # checksum, plaquette, trace checked
    assert dims == tuple(int(d) for d in lat400["dims"])
    ref = lat400["links"]
    # the stored rows bit for bit; the completed row as GLU's arithmetic
    # (which may fuse products) to an ulp
    assert np.array_equal(U[:, :, :2], ref[:, :, :2])
    assert np.abs(U[:, :, 2] - ref[:, :, 2]).max() <= 4e-16
    assert hdr["CHECKSUM"] == "f2ee7c36"


def test_write_reproduces_the_payload(lat400, tmp_path):
    out = tmp_path / "w.nersc"
    dims = tuple(int(d) for d in lat400["dims"])
    hdr = nersc.write(out, lat400["links"], dims, sequence_number=400)
    ref = FILE.read_bytes()
    _, off_ref = nersc.parse_header(ref)
    got = out.read_bytes()
    _, off = nersc.parse_header(got)
    assert got[off:] == ref[off_ref:]
    assert hdr["CHECKSUM"] == "f2ee7c36"


@pytest.mark.parametrize("datatype,fp", [("4D_SU3_GAUGE_3x3", "IEEE64BIG"),
                                         ("4D_SU3_GAUGE", "IEEE64LITTLE"),
                                         ("4D_SU3_GAUGE", "IEEE32BIG"),
                                         ("4D_SU3_GAUGE_3x3", "IEEE32LITTLE")])
def test_round_trips(hb8, tmp_path, datatype, fp):
    dims = tuple(int(d) for d in hb8["dims"])
    out = tmp_path / "r.nersc"
    nersc.write(out, hb8["links"], dims, datatype, fp)
    U, d2, _ = nersc.read(out)
    assert d2 == dims
    tol = 0.0 if (fp.startswith("IEEE64") and datatype.endswith("3x3")) else (
        4e-16 if fp.startswith("IEEE64") else 3e-7)
    assert np.abs(U - hb8["links"]).max() <= tol


def test_corrupted_payload_fails_the_checksum(tmp_path):
    data = bytearray(FILE.read_bytes())
    _, off = nersc.parse_header(bytes(data))
    data[off + 1000] ^= 0x10
    bad = tmp_path / "bad.nersc"
    bad.write_bytes(bytes(data))
    with pytest.raises(nersc.NerscError):
        nersc.read(bad)


ILDG = Path(__file__).resolve().parent / "golden" / "lat400.ildg"


def test_ildg_read_matches_glu(lat400):
    from glu_b200 import ildg
    U, dims, info = ildg.read(ILDG)  # SciDAC checksums verified
    assert dims == tuple(int(d) for d in lat400["dims"])
    assert np.array_equal(U, lat400["ildg_links"])
    assert (info["suma"], info["sumb"]) == (0xD00BA925, 0xC215FD4E)


@pytest.mark.parametrize("precision", [64, 32])
def test_ildg_write_round_trip(hb8, tmp_path, precision):
    from glu_b200 import ildg
    dims = tuple(int(d) for d in hb8["dims"])
    out = tmp_path / "w.ildg"
    ildg.write(out, hb8["links"], dims, precision)
    U, d2, info = ildg.read(out)
    assert d2 == dims and info["precision"] == precision
    tol = 0.0 if precision == 64 else 3e-7
    assert np.abs(U - hb8["links"]).max() <= tol


def test_glu_reads_our_ildg_file(reference, lat400, tmp_path):
    """GLU's own reader on a file written by ildg.write (the reference build
    travels with the repository as oracle/_ref)."""
    from glu_b200 import ildg
    dims = tuple(int(d) for d in lat400["dims"])
    out = tmp_path / "ours.ildg"
    ildg.write(out, lat400["ildg_links"], dims)
    back = reference.read_file(out, ildg=True)
    assert np.array_equal(back, lat400["ildg_links"])
