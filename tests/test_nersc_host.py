"""Host side of the NERSC codec: header parsing and the checksum convention
(no GPU)."""
from pathlib import Path

import numpy as np

from glu_b200.nersc import parse_header

FILE = Path(__file__).resolve().parent / "golden" / "lat400.nersc"


def test_header_and_checksum_of_the_fixture_file():
    data = FILE.read_bytes()
    hdr, off = parse_header(data)
    dims = tuple(int(hdr[f"DIMENSION_{k}"]) for k in range(1, 5))
    assert dims == (4, 4, 4, 8) and hdr["FLOATING_POINT"] == "IEEE64BIG"
    vals = np.frombuffer(data[off:], dtype=">f8")
    assert vals.size == int(np.prod(dims)) * 4 * 12
    # NERSC checksum: 32-bit wrapping sum of the host-order words
    words = np.frombuffer(vals.astype("<f8").tobytes(), dtype="<u4")
    assert int(words.sum(dtype=np.uint64) & 0xFFFFFFFF) == int(hdr["CHECKSUM"], 16)


def test_ildg_records_and_scidac_checksum_of_the_fixture_file():
    """LIME records of GLU's ILDG file and the SciDAC checksum convention
    (per-site CRC-32, rotated by site % 29 / % 31, XORed), in numpy."""
    import re
    import zlib

    from glu_b200.ildg import _record, parse_lime
    data = (FILE.parent / "lat400.ildg").read_bytes()
    recs = parse_lime(data)
    names = [n for n, _, _ in recs]
    assert "ildg-format" in names and "ildg-binary-data" in names
    pay = _record(data, recs, "ildg-binary-data")
    ck = _record(data, recs, "scidac-checksum").decode()
    suma = int(re.search(r"<suma>(\w+)</suma>", ck).group(1), 16)
    sumb = int(re.search(r"<sumb>(\w+)</sumb>", ck).group(1), 16)
    a = b = 0
    site = 4 * 18 * 8
    for i in range(len(pay) // site):
        c = zlib.crc32(pay[i * site:(i + 1) * site]) & 0xFFFFFFFF
        for r, acc in ((i % 29, "a"), (i % 31, "b")):
            v = ((c << r) | (c >> (32 - r))) & 0xFFFFFFFF if r else c
            if acc == "a":
                a ^= v
            else:
                b ^= v
    assert (a, b) == (suma, sumb)
