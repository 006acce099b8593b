// Layout mirrors of the GLU types the drop-in entry points read
// (src/Headers/GLU_types.h, default build: NC = 3, ND = 4, double
// precision, FFTW present).  Field order and types follow GLU exactly so
// that a pointer handed over by GLU can be read here.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace gfix {

// struct site (src/Headers/GLU_types.h:269-273)
struct glu_site {
  double **O;  // GLU_complex **O: O[mu] -> 9 complex, row-major
  size_t neighbor[4];
  size_t back[4];
};

// struct fftw_stuff (src/Headers/GLU_types.h:126-137)
struct glu_fftw_stuff {
  double **out;  // GLU_complex **
  double **in;   // GLU_complex **
  void *forward;
  void *backward;
  double *psq;
};

// struct latt_info (src/Headers/GLU_types.h:229-243)
struct glu_latt_info {
  size_t dims[4];
  size_t Lsq;
  size_t Lcu;
  size_t Volume;
  size_t flow;
  double gf_alpha;
  double sm_alpha[3];
  int head;  // header_mode enum
  uint32_t Seed[1];
  double twiddles[4];
  uint32_t Nthreads;
  void *su2_data;
  int argc;  // cline_arg enum
};

}  // namespace gfix

// struct cut_info (src/Headers/GLU_types.h:94-103), under GLU's own name: it
// is passed by value to cuts_struct, whose C declaration names it
struct cut_info {
  int dir;          // cut_mode
  int type;         // momentum_cut_def
  size_t max_mom;
  size_t max_t;
  char where[256];
  int definition;   // lie_field_def
  size_t angle;
  double cyl_width;
};
