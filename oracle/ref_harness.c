/*
 * ctypes-callable harness around the REFERENCE's own gauge-fixing code
 * (GLU compiled unmodified from its sources by oracle/Makefile).
 *
 * Test infrastructure only: used by the tests to pin the oracle, by the
 * golden-fixture script, and by the CPU-baseline timing.  It calls
 * GLU's FACG/FASD (src/Gfix/FACG.c:341-446), Coulomb_FA
 * (src/Gfix/CFACG.c:531-636), Landau (src/Gfix/Landau.c:261-374) and
 * Coulomb (src/Gfix/Coulomb.c:32-106) exactly as GLU's drivers do, and
 * records per-iteration trajectories through the FFTW stand-in's execute
 * hook (no reference source is patched).
 *
 * Host link layout at this boundary: double[V][ND][NC*NC][2] (site index
 * x fastest, then mu, then a row-major 3x3 complex matrix), which is GLU's
 * in-memory order of lat[i].O[mu][a*NC+b].
 */
#include "Mainfile.h"

#include "CFACG.h"
#include "Coulomb.h"
#include "FACG.h"
#include "GLUlib_wrap.h"
#include "cut_output.h"
#include "draughtboard.h"
#include "hb.h"
#include "par_rng.h"
#include "relax.h"
#include "cut_routines.h"
#include "cuts.h"
#include "Landau.h"
#include "geometry.h"
#include "init.h"
#include "gftests.h"
#include "plan_ffts.h"
#include "plaqs_links.h"
#include "random_config.h"

#include <omp.h>
#include <string.h>
#include <unistd.h>

/* GLU's global lattice description (src/Run/Mainfile.c:30) */
struct latt_info Latt;

static struct site *g_lat = NULL;

typedef struct {
  struct fftw_stuff *F;
  int coulomb;
  double *theta, *func;
  size_t cap, len;
} traj_t;

static traj_t g_traj;

static void free_lattice(void) {
  if (g_lat) free_lat(g_lat);
  g_lat = NULL;
}

static void set_threads(int nthreads) {
  omp_set_dynamic(0);
  omp_set_num_threads(nthreads > 0 ? nthreads : 1);
}

/* set up Latt for dims (x fastest) and allocate a unit-gauge lattice */
int ref_setup(const size_t *dims, int nthreads, double gf_alpha,
              unsigned seed) {
  free_lattice();
  set_threads(nthreads);
  for (int mu = 0; mu < ND; mu++) Latt.dims[mu] = dims[mu];
  Latt.gf_alpha = gf_alpha;
  Latt.Seed[0] = seed;
  Latt.head = UNIT_GAUGE;
  init_latt();
  if ((g_lat = allocate_lat()) == NULL) return -1;
  return 0;
}

/* read a configuration file with GLU's own reader; dims are returned.
 * head: 0 NERSC, 1 ILDG (SciDAC LIME) */
int ref_read_file_as(const char *path, size_t *dims_out, int nthreads, int head) {
  free_lattice();
  set_threads(nthreads);
  Latt.head = head == 1 ? ILDG_SCIDAC_HEADER : NERSC_HEADER;
  Latt.Seed[0] = 1;
  struct head_data HEAD;
  g_lat = read_file(&HEAD, path);
  if (g_lat == NULL) return -1;
  for (int mu = 0; mu < ND; mu++) dims_out[mu] = Latt.dims[mu];
  return 0;
}
int ref_read_file(const char *path, size_t *dims_out, int nthreads) {
  return ref_read_file_as(path, dims_out, nthreads, 0);
}

void ref_set_alpha(double gf_alpha) { Latt.gf_alpha = gf_alpha; }

/* change the OpenMP team size as init_latt would have recorded it
 * (src/Geometry/init.c:70-76) */
void ref_set_threads(int nthreads) {
  set_threads(nthreads);
#pragma omp parallel
  {
#pragma omp master
    Latt.Nthreads = (uint32_t)omp_get_num_threads();
  }
}

size_t ref_volume(void) { return Latt.Volume; }

int ref_put_links(const double *aos) {
  if (!g_lat) return -1;
  const size_t V = Latt.Volume;
#pragma omp parallel for
  for (size_t i = 0; i < V; i++)
    for (int mu = 0; mu < ND; mu++)
      memcpy(g_lat[i].O[mu], aos + ((i * ND + mu) * NCNC) * 2,
             NCNC * sizeof(GLU_complex));
  return 0;
}

int ref_get_links(double *aos) {
  if (!g_lat) return -1;
  const size_t V = Latt.Volume;
#pragma omp parallel for
  for (size_t i = 0; i < V; i++)
    for (int mu = 0; mu < ND; mu++)
      memcpy(aos + ((i * ND + mu) * NCNC) * 2, g_lat[i].O[mu],
             NCNC * sizeof(GLU_complex));
  return 0;
}

double ref_theta_test_lin(void) {
  GLU_real max;
  return theta_test_lin(g_lat, &max, ND);
}
double ref_gauge_functional(void) { return gauge_functional(g_lat); }
double ref_av_plaquette(void) { return av_plaquette(g_lat); }
void ref_latt_reunitU(void) { latt_reunitU(g_lat); }

/* post-fix diagnostics of GLU's output (Landau.c:42-66, Coulomb.c:37-41):
 * all_links, indivlinks (src/Field/plaqs_links.c:399-446), const_time
 * (src/Gfix/gftests.c:35-129) */
double ref_all_links(double *sp_link, double *t_link) {
  return all_links(g_lat, sp_link, t_link);
}
double ref_indivlinks(double *max) {
  GLU_real m = 0.0;
  const double avg = indivlinks(g_lat, &m);
  *max = (double)m;
  return avg;
}
void ref_const_time(double *lin, double *lg) { const_time(g_lat, lin, lg); }

/* the numbers of GLU's gf_check report (src/Wrappers/OBS_wrap.c:93-126):
 * theta_test_lin / _log with their maxima over ND and ND - 1 directions,
 * and const_time; out[10] in the order the report prints them */
void ref_gf_check(double *out) {
  GLU_real mx = 0.;
  out[0] = theta_test_lin(g_lat, &mx, ND);
  out[1] = mx;
  out[2] = theta_test_log(g_lat, &mx, ND);
  out[3] = mx;
  const_time(g_lat, &out[4], &out[5]);
  out[6] = theta_test_lin(g_lat, &mx, ND - 1);
  out[7] = mx;
  out[8] = theta_test_log(g_lat, &mx, ND - 1);
  out[9] = mx;
}

/* GLU's writer (src/IO/writers.c:329-420, write_configuration): storage
 * is a GLU_output value (OUTPUT_ILDG, OUTPUT_GAUGE, ...) */
int ref_write_config(const char *path, int storage, const char *details) {
  return write_configuration(g_lat, path, (GLU_output)storage, details);
}
int ref_output_code(const char *name) {
  if (!strcmp(name, "ILDG")) return OUTPUT_ILDG;
  if (!strcmp(name, "SCIDAC")) return OUTPUT_SCIDAC;
  if (!strcmp(name, "NERSC_GAUGE")) return OUTPUT_GAUGE;
  if (!strcmp(name, "NERSC_NCxNC")) return OUTPUT_NCxNC;
  return -1;
}

double ref_fft_seconds(void) { return glu_shim_fft_seconds(); }
void ref_reset_fft_seconds(void) { glu_shim_reset_fft_seconds(); }

/*
 * Landau: at the start of each FFT round (forward plan of field 0, before
 * it runs) the four `in` fields hold the packed derivative of the current
 * links (src/Gfix/FACG.c:57-60).  Undo the packing to recover the local
 * tr(dA dA) of src/Gfix/lin_derivs.c:181-185 and normalise with
 * GFNORM_LANDAU, which is the in-loop theta of src/Gfix/FACG.c:288-291.
 * Coulomb: after the backward plan of field 3 the `in` fields hold the
 * accelerated derivative, whose sum_DER2/sum_PR norm is the slice theta
 * (src/Gfix/CFACG.c:309-315, 347).  One thread only (fields run in order).
 */
static void traj_hook(void *ctx, fftw_plan p, int when, int sign, void *in,
                      void *out) {
  (void)sign; (void)in; (void)out;
  traj_t *T = (traj_t *)ctx;
  if (T->len >= T->cap) return;
  GLU_complex **f = T->F->in;
  if (!T->coulomb) {
    if (when != 0 || p != ((fftw_plan *)T->F->forward)[0]) return;
    double tr = 0.0, re = 0.0;
    for (size_t i = 0; i < LVOLUME; i++) {
      const double R0 = 3.0 * cimag(f[0][i]), R3 = -3.0 * creal(f[0][i]);
      const double R1 = 2.0 * creal(f[1][i]), I1 = 2.0 * cimag(f[1][i]);
      const double R2 = 2.0 * creal(f[2][i]), I2 = 2.0 * cimag(f[2][i]);
      const double R4 = 2.0 * creal(f[3][i]), I4 = 2.0 * cimag(f[3][i]);
      tr += 0.4444444444444444 * (R0 * R0 + R3 * (R3 + R0)) +
            (R1 * R1 + I1 * I1 + R2 * R2 + I2 * I2 + R4 * R4 + I4 * I4);
      for (int mu = 0; mu < ND; mu++)
        re += creal(g_lat[i].O[mu][0]) + creal(g_lat[i].O[mu][4]) +
              creal(g_lat[i].O[mu][8]);
    }
    T->theta[T->len] = tr * GFNORM_LANDAU;
    if (T->func) T->func[T->len] = 1.0 - re / (double)(ND * NC * LVOLUME);
    T->len++;
  } else {
    if (when != 1 || p != ((fftw_plan *)T->F->backward)[TRUE_HERM - 1])
      return;
    double s = 0.0;
    for (size_t i = 0; i < LCU; i++) {
      const double a = creal(f[0][i]), b = cimag(f[0][i]);
      double l = a * a + b * b + a * b;
      for (int k = 1; k < TRUE_HERM; k++)
        l += creal(f[k][i]) * creal(f[k][i]) + cimag(f[k][i]) * cimag(f[k][i]);
      s += 2.0 * l;
    }
    T->theta[T->len] = s * GFNORM_COULOMB;
    if (T->func) T->func[T->len] = 0.0;
    T->len++;
  }
}

static void arm_trajectory(struct fftw_stuff *F, int coulomb, double *theta,
                           double *func, size_t cap) {
  g_traj.F = F;
  g_traj.coulomb = coulomb;
  g_traj.theta = theta;
  g_traj.func = func;
  g_traj.cap = cap;
  g_traj.len = 0;
  if (theta && cap > 0 && Latt.Nthreads == 1)
    glu_shim_set_hook(traj_hook, &g_traj);
  else
    glu_shim_set_hook(NULL, NULL);
}

/* Landau FA solve: algo 0 = FACG, 1 = FASD (src/Gfix/FACG.c:341,395) with
 * the FFTW plans and p^2 table built as src/Gfix/Landau.c:272-284 does. */
size_t ref_landau_fa(int algo, double acc, size_t max_iters, double *th,
                     double *traj_theta, double *traj_func, size_t cap,
                     size_t *traj_len) {
  struct fftw_stuff FFTW;
  create_plans_DFT(&FFTW, Latt.dims, TRUE_HERM, ND);
  FFTW.psq = malloc(LVOLUME * sizeof(GLU_real));
  for (size_t i = 0; i < LVOLUME; i++)
    FFTW.psq[i] = MAX_LANDAU / (gen_p_sq(i, ND));
  arm_trajectory(&FFTW, 0, traj_theta, traj_func, cap);
  size_t iters = (algo == 0) ? FACG(g_lat, &FFTW, th, acc, max_iters)
                             : FASD(g_lat, &FFTW, th, acc, max_iters);
  glu_shim_set_hook(NULL, NULL);
  if (traj_len) *traj_len = g_traj.len;
  clean_up_fftw(FFTW, TRUE_HERM);
  return iters;
}

/* Coulomb FA solve (src/Gfix/CFACG.c:531) with the 3D plans and p^2 table
 * of src/Gfix/Coulomb.c:48-59; no final reunitarisation (that is in
 * Coulomb(), see ref_coulomb). */
size_t ref_coulomb_fa(int facg, double acc, size_t max_iters,
                      double *traj_theta, size_t cap, size_t *traj_len) {
  struct fftw_stuff FFTW;
  create_plans_DFT(&FFTW, Latt.dims, TRUE_HERM, ND - 1);
  FFTW.psq = malloc(LCU * sizeof(GLU_real));
  for (size_t i = 0; i < LCU; i++)
    FFTW.psq[i] = MAX_COULOMB / (gen_p_sq(i, ND - 1));
  arm_trajectory(&FFTW, 1, traj_theta, NULL, cap);
  size_t iters =
      Coulomb_FA(g_lat, &FFTW, acc, max_iters, facg ? GLU_TRUE : GLU_FALSE);
  glu_shim_set_hook(NULL, NULL);
  if (traj_len) *traj_len = g_traj.len;
  clean_up_fftw(FFTW, TRUE_HERM);
  return iters;
}

/* the full drivers, as GF_wrap calls them (src/Wrappers/GF_wrap.c:55,78) */
size_t ref_landau(double acc, size_t max_iters, const char *infile) {
  return Landau(g_lat, acc, max_iters, infile);
}

size_t ref_coulomb(double acc, size_t max_iters) {
  return Coulomb(g_lat, acc, max_iters);
}

/* momentum-space cuts (src/Cuts/cuts.c:110-184, cuts_struct) */
static struct cut_info cut_info_of(int dir, int type, size_t max_mom,
                                   int definition, size_t angle,
                                   double cyl_width) {
  struct cut_info c;
  memset(&c, 0, sizeof c);
  c.dir = (cut_mode)dir;
  c.type = (momentum_cut_def)type;
  c.max_mom = max_mom;
  c.definition = (lie_field_def)definition;
  c.angle = angle;
  c.cyl_width = cyl_width;
  return c;
}

/* compute_veclist (src/Cuts/cut_routines.c:459) in momentum space: the
 * number of momenta; up to cap entries of MOM (4 ints each) and idx */
long ref_veclist(int dir, int type, size_t max_mom, size_t angle,
                 double cyl_width, int *mom, size_t *idx, size_t cap) {
  struct cut_info c = cut_info_of(dir, type, max_mom, LINEAR_DEF, angle,
                                  cyl_width);
  if (c.dir == NONEXCEPTIONAL) c.type = PSQ_CUT;
  size_t n = 0;
  struct veclist *list = compute_veclist(&n, c, ND, GLU_FALSE);
  if (list == NULL) return 0;
  for (size_t i = 0; i < n && i < cap; i++) {
    for (int mu = 0; mu < ND; mu++) mom[i * ND + mu] = list[i].MOM[mu];
    idx[i] = list[i].idx;
  }
  free(list);
  return (long)n;
}

/* GLU's output file name for these cuts (src/Cuts/cut_output.c:121) */
int ref_cut_output_name(int dir, int type, size_t max_mom, int definition,
                        size_t angle, double cyl_width, size_t flow,
                        char *out, size_t cap) {
  struct cut_info c = cut_info_of(dir, type, max_mom, definition, angle,
                                  cyl_width);
  Latt.flow = flow;
  char *s = output_str_struct(c);
  snprintf(out, cap, "%s", s);
  free(s);
  return 0;
}

/* the whole measurement: writes GLU's output file into directory `where`
 * (GLU's default build writes to "./"); the lattice is left holding the
 * Fourier-transformed Lie fields, as in GLU */
int ref_cuts(int dir, int type, size_t max_mom, int definition, size_t angle,
             double cyl_width, size_t flow, const char *where) {
  struct cut_info c = cut_info_of(dir, type, max_mom, definition, angle,
                                  cyl_width);
  Latt.flow = flow;
  char cwd[4096];
  if (getcwd(cwd, sizeof cwd) == NULL || chdir(where) != 0) return -1;
  const int rc = cuts_struct(g_lat, c);
  if (chdir(cwd) != 0) return -1;
  return rc == GLU_SUCCESS ? 0 : -1;
}

/* configuration generation: GLU's over-relaxation sweeps (OR_lattice,
 * src/Update/relax.c:83-114) and heatbath steps (update_lattice,
 * src/Update/KPHB.c:83-99: hb_lattice then n_or OR_lattice) on the lattice
 * in place, with GLU's draughtboard (src/Geometry/draughtboard.c) and its
 * own generator seeded from Latt.Seed; plaq (may be NULL) receives the
 * average plaquette after every step */
/* GLU's sweeps use orphaned `omp for` loops: as in hb_update
 * (KPHB.c:193-250) they run inside one parallel region */
int ref_overrelax(size_t sweeps) {
  struct draughtboard db;
  if (!g_lat || init_cb(&db, LVOLUME, ND) == GLU_FAILURE) return -1;
#pragma omp parallel
  {
    for (size_t k = 0; k < sweeps; k++) OR_lattice(g_lat, db);
  }
  free_cb(&db);
  return 0;
}

int ref_heatbath(double beta, size_t iterations, size_t n_or, double *plaq) {
  struct draughtboard db;
  if (!g_lat || initialise_par_rng(NULL) == GLU_FAILURE) return -1;
  if (init_cb(&db, LVOLUME, ND) == GLU_FAILURE) return -1;
  const double inverse_beta = NC / beta;
#pragma omp parallel
  {
    for (size_t i = 0; i < iterations; i++) {
      hb_lattice(g_lat, inverse_beta, db);
      for (size_t k = 0; k < n_or; k++) OR_lattice(g_lat, db);
#pragma omp single
      {
        if (plaq) plaq[i] = av_plaquette(g_lat);
      }
    }
  }
  free_cb(&db);
  free_par_rng();
  return 0;
}
