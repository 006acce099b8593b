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
