"""Momentum-space gluon measurements through the GPU library: GLU's
cuts_struct (src/Cuts/cuts.c:110-184) for CUTTYPE = GLUON_PROPS,
EXCEPTIONAL and FIELDS, with GLU's input-file vocabulary
(src/IO/input_reader.c:354-431: CUTTYPE, MOM_CUT, FIELD_DEFINITION, MAXMOM,
ANGLE, CYL_WIDTH) and GLU's binary output file (src/Cuts/cut_output.c).

The momentum list (src/Cuts/cut_routines.c) is host code inside the
library; the Lie fields, their Fourier transforms, the p-space Landau
correction and the contractions run on the GPU.
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib

# GLU's enum values (src/Headers/GLU_enum.h)
CUTTYPES = {"EXCEPTIONAL": 0, "FIELDS": 2, "GLUON_PROPS": 6}
MOM_CUTS = {"HYPERCUBIC_CUT": 0, "SPHERICAL_CUT": 1, "CYLINDER_CUT": 2,
            "CONICAL_CUT": 3}
FIELD_DEFINITIONS = {"LINEAR": 0, "LOGARITHMIC": 1}


class CutsError(RuntimeError):
    pass


@dataclass
class CutInfo:
    """GLU's struct cut_info for the momentum-space modes, by input-file
    names; unknown MOM_CUT falls back to SPHERICAL_CUT as GLU's reader does."""
    cuttype: str = "GLUON_PROPS"
    mom_cut: str = "SPHERICAL_CUT"
    field_definition: str = "LINEAR"
    maxmom: int = 20
    angle: int = 60
    cyl_width: float = 2.0

    def c(self) -> _lib.GfixCutInfo:
        if self.cuttype not in CUTTYPES:
            raise CutsError(f"CUTTYPE {self.cuttype} not provided "
                            f"({', '.join(CUTTYPES)})")
        return _lib.GfixCutInfo(CUTTYPES[self.cuttype],
                                MOM_CUTS.get(self.mom_cut, 1), int(self.maxmom),
                                FIELD_DEFINITIONS.get(self.field_definition, 0),
                                int(self.angle), float(self.cyl_width))


def _dims(dims):
    return (C.c_size_t * 4)(*[int(d) for d in dims])


def _err(lib) -> str:
    return lib.gfix_cuts_error().decode()


def veclist(dims, info: CutInfo) -> np.ndarray:
    """The kept momenta (n, 4) in GLU's order."""
    lib = _lib.load()
    ci = info.c()
    n = lib.gfix_cut_veclist(_dims(dims), C.byref(ci), None, 0)
    if n < 0:
        raise CutsError(_err(lib))
    mom = np.zeros((max(n, 1), 4), dtype=np.int32)
    lib.gfix_cut_veclist(_dims(dims), C.byref(ci),
                         mom.ctypes.data_as(C.POINTER(C.c_int32)), n)
    return mom[:n]


def _outputs(info: CutInfo, n: int):
    if info.cuttype == "FIELDS":
        return np.zeros((n, 4, 3, 3), dtype=np.complex128), None
    return np.zeros(n), np.zeros(n)


def _result(info, mom, o0, o1, err):
    out = {"mom": mom, "pspace_err": float(err)}
    if info.cuttype == "GLUON_PROPS":
        out.update(transverse=o0, longitudinal=o1)
    elif info.cuttype == "EXCEPTIONAL":
        out.update(g2=o0, g3=o1)
    else:
        out.update(fields=o0)
    return out


def measure(links, dims, info: CutInfo) -> dict:
    """The measurement of cuts_struct on host links (V, 4, 3, 3): mom and
    transverse/longitudinal (GLUON_PROPS), g2/g3 (EXCEPTIONAL) or fields
    (FIELDS), plus the p-space gauge error."""
    lib = _lib.load()
    U = np.ascontiguousarray(links, dtype=np.complex128)
    mom = veclist(dims, info)
    o0, o1 = _outputs(info, len(mom))
    e = C.c_double(0.0)
    rc = lib.gfix_cuts_measure(U.ctypes.data, _dims(dims), C.byref(info.c()), len(mom),
                               o0.ctypes.data_as(_lib._dp),
                               o1.ctypes.data_as(_lib._dp) if o1 is not None else None,
                               C.byref(e))
    if rc != 0:
        raise CutsError(_err(lib))
    return _result(info, mom, o0, o1, e.value)


def measure_device(links, dims, info: CutInfo) -> dict:
    """The same on links already in device memory: a CUDA tensor of GLU's
    layout (any dtype view of double[V][4][9][2])."""
    lib = _lib.load()
    mom = veclist(dims, info)
    o0, o1 = _outputs(info, len(mom))
    e = C.c_double(0.0)
    rc = lib.gfix_cuts_measure_device(links.data_ptr(), _dims(dims), C.byref(info.c()),
                                      len(mom), o0.ctypes.data_as(_lib._dp),
                                      o1.ctypes.data_as(_lib._dp) if o1 is not None
                                      else None, C.byref(e))
    if rc != 0:
        raise CutsError(_err(lib))
    return _result(info, mom, o0, o1, e.value)


def cuts_struct(links, dims, info: CutInfo, where: str = "./", flow: int = 0):
    """GLU's cuts_struct: measure and write GLU's output file; returns
    (path, p-space error)."""
    lib = _lib.load()
    U = np.ascontiguousarray(links, dtype=np.complex128)
    e = C.c_double(0.0)
    buf = C.create_string_buffer(4096)
    rc = lib.gfix_cuts_write(U.ctypes.data, _dims(dims), C.byref(info.c()),
                             str(where).encode(), int(flow), C.byref(e), buf, 4096)
    if rc != 0:
        raise CutsError(_err(lib))
    return Path(buf.value.decode()), e.value


def read_output(path, cuttype: str = "GLUON_PROPS") -> dict:
    """Parse a GLU cut output file (big-endian): the momentum list
    (write_mom_veclist) then two lists (write_g2g3_to_list) or the fields
    (write_lattice_fields)."""
    d = Path(path).read_bytes()
    n = struct.unpack(">i", d[:4])[0]
    pos = 4
    k = np.frombuffer(d[pos:pos + 20 * n], dtype=">i4").reshape(n, 5).astype(np.int64)
    pos += 20 * n
    if (k[:, 0] != 4).any():
        raise CutsError("momentum records without dimension 4")
    out = {"mom": k[:, 1:]}
    n2 = struct.unpack(">I", d[pos:pos + 4])[0]
    pos += 4
    if cuttype == "FIELDS":
        a = np.frombuffer(d[pos:pos + 8 * 72 * n2], dtype=">f8").astype(np.float64)
        out["fields"] = a.view(np.complex128).reshape(n2, 4, 3, 3)
        pos += 8 * 72 * n2
    else:
        a = np.frombuffer(d[pos:pos + 8 * n2], dtype=">f8").astype(np.float64)
        pos += 8 * n2
        n3 = struct.unpack(">I", d[pos:pos + 4])[0]
        pos += 4
        b = np.frombuffer(d[pos:pos + 8 * n3], dtype=">f8").astype(np.float64)
        pos += 8 * n3
        names = ("transverse", "longitudinal") if cuttype == "GLUON_PROPS" else ("g2", "g3")
        out.update({names[0]: a, names[1]: b})
    if pos != len(d):
        raise CutsError(f"{len(d) - pos} trailing bytes in {path}")
    return out
