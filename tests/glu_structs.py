"""ctypes mirrors of the GLU types the GLU-named entry points read, for
tests that call them as GLU does (a struct site lattice, the global Latt).

Layouts: src/Headers/GLU_types.h (default build: NC = 3, ND = 4, double
precision, FFTW present).
"""
import ctypes as C

import numpy as np


class Site(C.Structure):
    """struct site (src/Headers/GLU_types.h:269-273)"""
    _fields_ = [("O", C.POINTER(C.POINTER(C.c_double))),
                ("neighbor", C.c_size_t * 4), ("back", C.c_size_t * 4)]


class Latt(C.Structure):
    """struct latt_info (src/Headers/GLU_types.h:229-243)"""
    _fields_ = [("dims", C.c_size_t * 4), ("Lsq", C.c_size_t), ("Lcu", C.c_size_t),
                ("Volume", C.c_size_t), ("flow", C.c_size_t), ("gf_alpha", C.c_double),
                ("sm_alpha", C.c_double * 3), ("head", C.c_int), ("Seed", C.c_uint32 * 1),
                ("twiddles", C.c_double * 4), ("Nthreads", C.c_uint32),
                ("su2_data", C.c_void_p), ("argc", C.c_int)]


class CutInfo(C.Structure):
    """struct cut_info (src/Headers/GLU_types.h:94-103)"""
    _fields_ = [("dir", C.c_int), ("type", C.c_int), ("max_mom", C.c_size_t),
                ("max_t", C.c_size_t), ("where", C.c_char * 256), ("definition", C.c_int),
                ("angle", C.c_size_t), ("cyl_width", C.c_double)]


class FftwStuff(C.Structure):
    """struct fftw_stuff (src/Headers/GLU_types.h:126-137)"""
    _fields_ = [("out", C.POINTER(C.POINTER(C.c_double))),
                ("inp", C.POINTER(C.POINTER(C.c_double))),
                ("forward", C.c_void_p), ("backward", C.c_void_p),
                ("psq", C.POINTER(C.c_double))]


class SiteLattice:
    """A GLU-style lattice over a numpy array of links (V, 4, 3, 3): each
    lat[i].O[mu] points into the array, which holds the links in place."""

    def __init__(self, links):
        self.U = np.ascontiguousarray(links, dtype=np.complex128).reshape(-1, 4, 3, 3).copy()
        V = self.U.shape[0]
        base = self.U.ctypes.data
        dp = C.POINTER(C.c_double)
        self._ptrs = [(dp * 4)(*[C.cast(base + (i * 4 + mu) * 144, dp) for mu in range(4)])
                      for i in range(V)]
        self.sites = (Site * V)()
        for i in range(V):
            self.sites[i].O = C.cast(self._ptrs[i], C.POINTER(dp))


def set_latt(lib, dims, gf_alpha=0.08, seed=1, flow=0):
    """Fill the library's Latt as GLU's init_latt would for these dims."""
    latt = Latt.in_dll(lib, "Latt")
    for mu in range(4):
        latt.dims[mu] = int(dims[mu])
    latt.Lsq = int(dims[0] * dims[1])
    latt.Lcu = int(dims[0] * dims[1] * dims[2])
    latt.Volume = int(np.prod(dims))
    latt.flow = flow
    latt.gf_alpha = gf_alpha
    latt.Seed[0] = seed
    return latt


def fftw_fields(fields):
    """struct fftw_stuff whose in[0..3] point at the rows of `fields`
    (complex128, shape (4, n)); returns (struct, keep-alive)."""
    f = np.ascontiguousarray(fields, dtype=np.complex128)
    dp = C.POINTER(C.c_double)
    rows = (dp * 4)(*[C.cast(f[k].ctypes.data, dp) for k in range(4)])
    st = FftwStuff()
    st.inp = C.cast(rows, C.POINTER(dp))
    return st, (f, rows)


def flush_c_stdio():
    """Flush the C library's stdio buffers (output of printf in the library)."""
    libc = C.CDLL(None)
    libc.fflush(None)


# GLU input file for its own program: gauge fixing of a NERSC configuration
# (GFTYPE LANDAU or COULOMB), with the other sections GLU's parser reads
GLU_INPUT = """MODE = GAUGE_FIXING
HEADER = NERSC
	DIM_0 = {d0}
	DIM_1 = {d1}
	DIM_2 = {d2}
	DIM_3 = {d3}
CONFNO = 400
RANDOM_TRANSFORM = NO
SEED = 0
GFTYPE = {gftype}
	GF_TUNE = {tune}
	ACCURACY = 14
	MAX_ITERS = {max_iters}
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
CONFIG_INFO = glu_b200_boundary_test
	STORAGE = NERSC_GAUGE
BETA = 6.0
	ITERS = 1500
	MEASURE = 1
	OVER_ITERS = 4
	SAVE = 25
	THERM = 100
"""
