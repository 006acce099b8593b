"""NERSC configuration files through the GPU codec (gfix_nersc_decode /
gfix_nersc_encode), GLU's I/O conventions (src/IO/read_headers.c:227-345,
src/IO/readers.c:169-310, src/IO/read_config.c:34-122).

A NERSC file is a text header between BEGIN_HEADER and END_HEADER lines of
``KEY = VALUE`` pairs, then the binary payload.  The header parsing and the
plaquette / link-trace checks are host work; the payload decode (byte order,
third-row completion, checksum) runs on the GPU.  Formats: DATATYPE
4D_SU3_GAUGE (12 reals per link) and 4D_SU3_GAUGE_3x3 (18); FLOATING_POINT
IEEE64BIG, IEEE32BIG (also IEEE32), IEEE64LITTLE, IEEE32LITTLE.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

# GLU's PLAQ_AND_TRACE_TOL (src/Headers/GLU_definitions.h): 1e-6
PLAQ_AND_TRACE_TOL = 1e-6

_FP = {"IEEE64BIG": (8, True), "IEEE32BIG": (4, True), "IEEE32": (4, True),
       "IEEE64LITTLE": (8, False), "IEEE32LITTLE": (4, False)}
_TYPES = {"4D_SU3_GAUGE": 12, "4D_SU3_GAUGE_3x3": 18}


class NerscError(RuntimeError):
    pass


def parse_header(data: bytes) -> tuple[dict, int]:
    """(header dict, payload offset)."""
    start = data.find(b"BEGIN_HEADER")
    end = data.find(b"END_HEADER")
    if start < 0 or end < 0:
        raise NerscError("no BEGIN_HEADER / END_HEADER")
    off = data.find(b"\n", end) + 1
    hdr = {}
    for line in data[start:end].decode("ascii", "replace").splitlines()[1:]:
        if "=" in line:
            k, v = line.split("=", 1)
            hdr[k.strip()] = v.strip()
    return hdr, off


def decode(payload: bytes, dims, nreal=12, bytes_per_real=8, big_endian=True):
    """(links (V, 4, 3, 3) complex128, checksum) of a raw payload."""
    lib = _lib.load()
    d = tuple(int(x) for x in dims)
    V = int(np.prod(d))
    need = V * 4 * nreal * bytes_per_real
    if len(payload) < need:
        raise NerscError(f"payload of {len(payload)} bytes, {need} needed")
    buf = np.frombuffer(payload, dtype=np.uint8, count=need)
    links = np.empty((V, 4, 3, 3), dtype=np.complex128)
    ck = C.c_uint32(0)
    rc = lib.gfix_nersc_decode(buf.ctypes.data, (C.c_size_t * 4)(*d), nreal,
                               bytes_per_real, int(big_endian), links.ctypes.data,
                               C.byref(ck))
    if rc != 0:
        raise NerscError(lib.gfix_nersc_error().decode())
    return links, int(ck.value)


def encode(links, dims, nreal=12, bytes_per_real=8, big_endian=True):
    """(payload bytes, checksum) of links (V, 4, 3, 3)."""
    lib = _lib.load()
    d = tuple(int(x) for x in dims)
    U = np.ascontiguousarray(links, dtype=np.complex128).reshape(-1, 4, 3, 3)
    out = np.empty(U.shape[0] * 4 * nreal * bytes_per_real, dtype=np.uint8)
    ck = C.c_uint32(0)
    rc = lib.gfix_nersc_encode(U.ctypes.data, (C.c_size_t * 4)(*d), nreal,
                               bytes_per_real, int(big_endian), out.ctypes.data,
                               C.byref(ck))
    if rc != 0:
        raise NerscError(lib.gfix_nersc_error().decode())
    return out.tobytes(), int(ck.value)


def read(path, check=True):
    """(links, dims, header) of a NERSC file; with check, the checksum,
    plaquette and link trace of the header are verified as GLU does."""
    from .gfix import link_diagnostics, observables
    data = open(path, "rb").read()
    hdr, off = parse_header(data)
    try:
        dims = tuple(int(hdr[f"DIMENSION_{k}"]) for k in range(1, 5))
        bytes_per_real, big = _FP[hdr["FLOATING_POINT"]]
        nreal = _TYPES[hdr["DATATYPE"]]
    except KeyError as e:
        raise NerscError(f"unsupported or missing header entry {e}") from None
    links, ck = decode(data[off:], dims, nreal, bytes_per_real, big)
    if check:
        want = int(hdr.get("CHECKSUM", "0"), 16)
        if ck != want:
            raise NerscError(f"checksum {ck:x} != header {want:x}")
        plaq = observables(links, dims)[2]
        tr = link_diagnostics(links, dims)["link"]
        if abs(plaq - float(hdr.get("PLAQUETTE", plaq))) > PLAQ_AND_TRACE_TOL:
            raise NerscError("plaquette differs from the header's")
        if abs(tr - float(hdr.get("LINK_TRACE", tr))) > PLAQ_AND_TRACE_TOL:
            raise NerscError("link trace differs from the header's")
    return links, dims, hdr


def write(path, links, dims, datatype="4D_SU3_GAUGE", floating_point="IEEE64BIG",
          ensemble_id="glu_b200", sequence_number=1):
    """A NERSC file of `links`; returns the header written."""
    from .gfix import link_diagnostics, observables
    bytes_per_real, big = _FP[floating_point]
    nreal = _TYPES[datatype]
    payload, ck = encode(links, dims, nreal, bytes_per_real, big)
    d = tuple(int(x) for x in dims)
    hdr = {"HDR_VERSION": "1.0", "DATATYPE": datatype, "STORAGE_FORMAT": "1.0"}
    for k in range(4):
        hdr[f"DIMENSION_{k + 1}"] = str(d[k])
    hdr["LINK_TRACE"] = "%1.15f" % link_diagnostics(links, d)["link"]
    hdr["PLAQUETTE"] = "%1.15f" % observables(links, d)[2]
    for k in range(4):
        hdr[f"BOUNDARY_{k + 1}"] = "PERIODIC"
    hdr["CHECKSUM"] = "%x" % ck
    hdr["ENSEMBLE_ID"] = ensemble_id
    hdr["SEQUENCE_NUMBER"] = str(int(sequence_number))
    hdr["FLOATING_POINT"] = floating_point
    text = "BEGIN_HEADER\n" + "".join(f"{k} = {v}\n" for k, v in hdr.items()) + "END_HEADER\n"
    with open(path, "wb") as f:
        f.write(text.encode("ascii"))
        f.write(payload)
    return hdr
