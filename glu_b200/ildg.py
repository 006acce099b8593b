"""ILDG (SciDAC LIME) configuration files through the GPU codec: the binary
record is GLU's full 3x3 big-endian payload (src/IO/Scidac.c,
src/IO/writers.c:329-420), decoded by gfix_nersc_decode (18 reals per link)
and checked against the scidac-checksum record with gfix_scidac_checksum.

A LIME file is a sequence of records, each a 144-byte big-endian header --
magic 0x456789ab (4 bytes), version (2), flags (2: message begin / end),
data length (8), type name (128, NUL-padded) -- then the data, padded to a
multiple of 8 bytes.  The LIME container, the XML records and the checks
are host work here.
"""
from __future__ import annotations

import ctypes as C
import re
import struct

import numpy as np

from . import _lib
from .nersc import NerscError, decode, encode

LIME_MAGIC = 0x456789AB


def parse_lime(data: bytes) -> list[tuple[str, int, int]]:
    """[(record type, data offset, data length)] of a LIME file."""
    out, pos = [], 0
    while pos + 144 <= len(data):
        magic, _ver, _flags, length = struct.unpack(">IHHQ", data[pos:pos + 16])
        if magic != LIME_MAGIC:
            raise NerscError(f"no LIME record at byte {pos}")
        name = data[pos + 16:pos + 144].split(b"\0", 1)[0].decode("ascii", "replace")
        out.append((name, pos + 144, length))
        pos += 144 + length + (-length % 8)
    return out


def _record(data, recs, name):
    for n, off, ln in recs:
        if n == name:
            return data[off:off + ln]
    return None


def scidac_checksum(payload: bytes, site_bytes: int, nsites: int) -> tuple[int, int]:
    lib = _lib.load()
    buf = np.frombuffer(payload, dtype=np.uint8, count=site_bytes * nsites)
    a, b = C.c_uint32(0), C.c_uint32(0)
    if lib.gfix_scidac_checksum(buf.ctypes.data, site_bytes, nsites, C.byref(a),
                                C.byref(b)) != 0:
        raise NerscError(lib.gfix_nersc_error().decode())
    return int(a.value), int(b.value)


def read(path, check=True):
    """(links, dims, info) of an ILDG file; with check, the SciDAC
    checksums of the binary record are verified."""
    data = open(path, "rb").read()
    recs = parse_lime(data)
    fmt = _record(data, recs, "ildg-format")
    payload = _record(data, recs, "ildg-binary-data")
    if fmt is None or payload is None:
        raise NerscError("ildg-format or ildg-binary-data record missing")
    fmt = fmt.decode("ascii", "replace")
    try:
        dims = tuple(int(re.search(rf"<{k}>\s*(\d+)\s*</{k}>", fmt).group(1))
                     for k in ("lx", "ly", "lz", "lt"))
        prec = int(re.search(r"<precision>\s*(\d+)\s*</precision>", fmt).group(1))
    except AttributeError:
        raise NerscError("ildg-format record without dimensions / precision") from None
    bpr = prec // 8
    links, _ = decode(payload, dims, 18, bpr, True)
    info = {"precision": prec}
    ck = _record(data, recs, "scidac-checksum")
    if ck is not None:
        t = ck.decode("ascii", "replace")
        suma = int(re.search(r"<suma>\s*([0-9a-fA-F]+)\s*</suma>", t).group(1), 16)
        sumb = int(re.search(r"<sumb>\s*([0-9a-fA-F]+)\s*</sumb>", t).group(1), 16)
        info.update(suma=suma, sumb=sumb)
        if check:
            a, b = scidac_checksum(payload, 4 * 18 * bpr, int(np.prod(dims)))
            if (a, b) != (suma, sumb):
                raise NerscError(f"SciDAC checksums {a:x} {b:x} != {suma:x} {sumb:x}")
    return links, dims, info


def _lime_record(name: str, data: bytes, flags: int) -> bytes:
    head = struct.pack(">IHHQ", LIME_MAGIC, 1, flags, len(data))
    head += name.encode("ascii").ljust(128, b"\0")
    return head + data + b"\0" * (-len(data) % 8)


def write(path, links, dims, precision=64):
    """An ILDG file of `links` (records as GLU writes them); returns the
    SciDAC checksums."""
    d = tuple(int(x) for x in dims)
    bpr = precision // 8
    payload, _ = encode(links, d, 18, bpr, True)
    a, b = scidac_checksum(payload, 4 * 18 * bpr, int(np.prod(d)))
    xml = '<?xml version="1.0" encoding="UTF-8"?>'
    recs = [
        ("scidac-private-file-xml",
         xml + "<scidacFile><version>1.1</version><spacetime>4</spacetime><dims>"
         + " ".join(map(str, d)) + "</dims><volfmt>0</volfmt></scidacFile>"),
        ("scidac-file-xml", "<title>glu_b200 ILDG gauge configuration</title>"),
        ("scidac-private-record-xml",
         xml + "<scidacRecord><version>1.0</version><globaldata>0</globaldata>"
         "<datatype>QDP_%s3_ColorMatrix</datatype><precision>%s</precision>"
         "<colors>3</colors><typesize>%d</typesize><datacount>4</datacount>"
         "</scidacRecord>" % ("D" if precision == 64 else "F",
                              "D" if precision == 64 else "F", 18 * bpr)),
        ("scidac-record-xml", "<info>glu_b200 configuration</info>"),
        ("ildg-format",
         xml + '<ildgFormat xmlns="http://www.lqcd.org/ildg"><version>1.0</version>'
         "<field>su3gauge</field><precision>%d</precision>"
         "<lx>%d</lx><ly>%d</ly><lz>%d</lz><lt>%d</lt></ildgFormat>" % ((precision,) + d)),
    ]
    out = b""
    for i, (n, t) in enumerate(recs):
        out += _lime_record(n, t.encode("ascii"), 0xC000 if i == 0 else 0)
    out += _lime_record("ildg-binary-data", payload, 0)
    ck = (xml + "<scidacChecksum><version>1.0</version><suma>%x</suma><sumb>%x</sumb>"
          "</scidacChecksum>" % (a, b))
    out += _lime_record("scidac-checksum", ck.encode("ascii"), 0x4000)
    with open(path, "wb") as f:
        f.write(out)
    return a, b
