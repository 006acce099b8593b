// GLU's gauge-fixing entry points on top of the flat gfix_* interface.
//
// The caller is GLU (or a program built like it): `lat` is GLU's AoS
// lattice, the lattice shape and GF_TUNE are read from GLU's global Latt.
// Each call gathers the links into one contiguous buffer, runs the GPU
// solve, scatters them back, and follows GLU's return conventions.
#include <cuda_runtime.h>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/glu_gfix.h"
#include "glu_compat.h"

namespace gfix {
void set_restart_log(bool on);  // gfix.cu: print GLU's restart messages
}

using gfix::glu_fftw_stuff;
using gfix::glu_latt_info;
using gfix::glu_site;

// GLU's global lattice description (src/Run/Mainfile.c:30).  Weak: inside
// the GLU program its own definition is the one every reference binds to.
extern "C" {
__attribute__((weak)) glu_latt_info Latt;
}

namespace {

constexpr size_t kGluFailure = (size_t)-1;  // GLU_FAILURE returned as size_t
constexpr int kGfGluFailures = 7;           // GF_GLU_FAILURES (GLU_definitions.h:400-402)

// optional precision selection for the drop-in entry points:
//   GLU_GFIX_PRECISION = FP64 (default) | MIXED
//   GLU_GFIX_SWITCH    = x  (FP32 until theta < 10^-x, default 9)
void env_precision(gfix_params *p) {
  p->precision = GFIX_FP64;
  p->switch_theta = 1e-9;
  if (const char *s = getenv("GLU_GFIX_PRECISION"))
    if (!strcmp(s, "MIXED") || !strcmp(s, "mixed")) p->precision = GFIX_MIXED;
  if (const char *s = getenv("GLU_GFIX_SWITCH")) {
    const double x = atof(s);
    if (x > 0) p->switch_theta = pow(10.0, -x);
  }
}

// GLU's compile-time Landau options, which a program linked against this
// library sets at run time instead (GLU's own #defines do not reach here):
//   GLU_GFIX_LUXURY   = N  (LUXURY_GAUGE: N random gauge copies per attempt)
//   GLU_GFIX_BEST_COPY = 1 (BEST_COPY: keep the copy of least functional)
void env_luxury(gfix_params *p) {
  p->luxury_copies = 0;
  p->luxury_best = 0;
  if (const char *s = getenv("GLU_GFIX_LUXURY")) p->luxury_copies = std::max(0, atoi(s));
  if (const char *s = getenv("GLU_GFIX_BEST_COPY")) p->luxury_best = atoi(s) != 0;
}

void dims_of(size_t *d) {
  for (int i = 0; i < 4; i++) d[i] = Latt.dims[i];
}

size_t volume() { return Latt.dims[0] * Latt.dims[1] * Latt.dims[2] * Latt.dims[3]; }

// lat[i].O[mu] (separate 144-byte allocations) <-> contiguous double[V][4][18]
void gather(const glu_site *lat, double *buf, size_t V) {
#pragma omp parallel for
  for (long long i = 0; i < (long long)V; i++)
    for (int mu = 0; mu < 4; mu++)
      memcpy(buf + ((size_t)i * 4 + mu) * 18, lat[i].O[mu], 18 * sizeof(double));
}

void scatter(glu_site *lat, const double *buf, size_t V) {
#pragma omp parallel for
  for (long long i = 0; i < (long long)V; i++)
    for (int mu = 0; mu < 4; mu++)
      memcpy(lat[i].O[mu], buf + ((size_t)i * 4 + mu) * 18, 18 * sizeof(double));
}

// One pinned staging buffer for the whole process, grown on demand: GLU
// calls these entry points once per configuration with the same lattice,
// and a fresh cudaMallocHost of the link payload per call costs more than
// the copies themselves.  Freed at exit.
struct Staging {
  double *p = nullptr;
  size_t n = 0;
  ~Staging() {
    if (p) cudaFreeHost(p);
  }
  double *get(size_t need) {
    if (need <= n) return p;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    if (cudaMallocHost(&p, need * sizeof(double)) != cudaSuccess) {
      p = nullptr;
      return nullptr;
    }
    n = need;
    return p;
  }
};
Staging g_stage;

struct Buf {
  double *p;
  explicit Buf(size_t n) : p(g_stage.get(n)) {}
};

size_t landau_fa(glu_site *lat, double *th, double acc, size_t max_iters,
                 int algo) {
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  Buf buf(V * 72);
  if (!buf.p) {
    fprintf(stderr, "[FACG] allocation of temporaries failed\n");
    return 0;
  }
  gather(lat, buf.p, V);
  gfix_params p;
  memset(&p, 0, sizeof p);
  p.gf_alpha = Latt.gf_alpha;
  p.accuracy = acc;
  p.max_iters = max_iters;
  p.algo = algo;
#ifdef GLU_GFIX_SD
  p.sd_fixed_step = 1;
#endif
  env_precision(&p);
  gfix_result r;
  if (gfix_landau(buf.p, d, &p, &r) != 0) {
    fprintf(stderr, "[GF] GPU gauge fixing failed: %s\n", gfix_last_error());
    return 0;
  }
  scatter(lat, buf.p, V);
  *th = r.theta;
  return r.iters;
}

}  // namespace

extern "C" {

size_t FACG(struct site *lat, struct fftw_stuff *FFTW, double *th,
            const double acc, const size_t max_iters) {
  (void)FFTW;
  return landau_fa(reinterpret_cast<glu_site *>(lat), th, acc, max_iters,
                   GFIX_CG);
}

size_t FASD(struct site *lat, struct fftw_stuff *FFTW, double *th,
            const double acc, const size_t max_iters) {
  (void)FFTW;
  return landau_fa(reinterpret_cast<glu_site *>(lat), th, acc, max_iters,
                   GFIX_SD);
}

void FOURIER_ACCELERATE3(struct fftw_stuff *FFTW) {
  glu_fftw_stuff *F = reinterpret_cast<glu_fftw_stuff *>(FFTW);
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  std::vector<double> f(V * 8);
  for (int k = 0; k < 4; k++)
    memcpy(f.data() + (size_t)k * V * 2, F->in[k], V * 2 * sizeof(double));
  if (gfix_fourier_accelerate(f.data(), d, 4) != 0) {
    fprintf(stderr, "[GF] GPU Fourier acceleration failed: %s\n",
            gfix_last_error());
    return;
  }
  for (int k = 0; k < 4; k++)
    memcpy(F->in[k], f.data() + (size_t)k * V * 2, V * 2 * sizeof(double));
}

size_t Landau(struct site *lat, const double accuracy, const size_t iter,
              const char *infile) {
  (void)infile;
  glu_site *L = reinterpret_cast<glu_site *>(lat);
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  Buf buf(V * 72);
  if (!buf.p) {
    fprintf(stderr, "[GF] allocation of the GPU staging buffer failed\n");
    return kGluFailure;
  }
  gather(L, buf.p, V);
  gfix_params p;
  memset(&p, 0, sizeof p);
  p.gf_alpha = Latt.gf_alpha;
  p.accuracy = accuracy;
  p.max_iters = iter;
  p.algo = GFIX_CG;
#ifdef GLU_GFIX_SD
  p.algo = GFIX_SD;
  p.sd_fixed_step = 1;
#endif
  // GLU's restart loop: up to GF_GLU_FAILURES - 1 random restarts
  // (src/Gfix/Landau.c:322), the transforms seeded by GLU's seed
  p.max_restarts = kGfGluFailures - 1;
  p.restart_seed = Latt.Seed[0];
  env_precision(&p);
  env_luxury(&p);
  gfix_result r;
  double obs[3] = {0, 0, 0}, dg[6] = {0, 0, 0, 0, 0, 0};
  gfix::set_restart_log(true);
  const int rc = gfix_landau_driver(buf.p, d, &p, &r, obs, dg);
  gfix::set_restart_log(false);
  if (rc != 0) {
    fprintf(stderr, "[GF] GPU gauge fixing failed: %s\n", gfix_last_error());
    return kGluFailure;
  }
  // the links of the last attempt go back to the caller either way
  scatter(L, buf.p, V);
  if (r.iters == kGluFailure) {
    printf("\n[GF] Failure to converge to a sufficient solution \n"
           "[GF] Please lower the GF_TUNE parameter from %g \n",
           Latt.gf_alpha);
    return kGluFailure;
  }
  // output_fixing_info (src/Gfix/Landau.c:42-66), computed on the GPU by
  // the driver: reunitarised links, plaquette, link traces, const_time,
  // functional
  printf("[GF] Plaquette :: %1.15f \n[GF] Accuracy :: %1.4e\n", obs[2],
         r.theta);
  printf("[GF] Iters :: %zu\n[GF] Link trace :: %1.15f || Maximum :: %1.15f\n",
         r.iters, dg[2], dg[3]);
  printf("[GF] Temporal constance || Lin %e || Log %e \n", dg[4], dg[5]);
  printf("[GF] Functional :: %1.15f\n", obs[1]);
  return r.iters;
}

size_t Coulomb_FA(struct site *lat, struct fftw_stuff *FFTW,
                  const double accuracy, const size_t max_iter,
                  const int FACG_flag) {
  (void)FFTW;
  glu_site *L = reinterpret_cast<glu_site *>(lat);
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  Buf buf(V * 72);
  if (!buf.p) {
    fprintf(stderr, "[CG] allocation of the GPU staging buffer failed\n");
    return 0;
  }
  gather(L, buf.p, V);
  gfix_params p;
  memset(&p, 0, sizeof p);
  p.gf_alpha = Latt.gf_alpha;
  p.accuracy = accuracy;
  p.max_iters = max_iter;
  p.algo = FACG_flag ? GFIX_CG : GFIX_SD;
#ifdef GLU_GFIX_SD
  p.sd_fixed_step = 1;
#endif
  env_precision(&p);
  gfix_result r;
  if (gfix_coulomb(buf.p, d, &p, &r, nullptr, nullptr) != 0) {
    fprintf(stderr, "[CG] GPU Coulomb gauge fixing failed: %s\n",
            gfix_last_error());
    return 0;
  }
  scatter(L, buf.p, V);
  return r.iters;
}

size_t Coulomb(struct site *lat, const double accuracy, const size_t iter) {
  glu_site *L = reinterpret_cast<glu_site *>(lat);
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  Buf buf(V * 72);
  if (!buf.p) {
    fprintf(stderr, "[CG] allocation of the GPU staging buffer failed\n");
    return 0;
  }
  gather(L, buf.p, V);
  gfix_params p;
  memset(&p, 0, sizeof p);
  p.gf_alpha = Latt.gf_alpha;
  p.accuracy = accuracy;
  p.max_iters = iter;
#ifdef GLU_GFIX_SD
  p.algo = GFIX_SD;
  p.sd_fixed_step = 1;
#else
  p.algo = GFIX_CG;
#endif
  env_precision(&p);
  // the initial link traces and plaquette, the solve of every slice, the
  // final latt_reunitU (src/Gfix/Coulomb.c:97) and the final diagnostics,
  // in one sequence on the GPU
  gfix_result r;
  double obs0[3] = {0, 0, 0}, dg0[6] = {0, 0, 0, 0, 0, 0};
  double obs[3] = {0, 0, 0}, dg[6] = {0, 0, 0, 0, 0, 0};
  if (gfix_coulomb_driver(buf.p, d, &p, &r, obs0, dg0, obs, dg) != 0) {
    fprintf(stderr, "[CG] GPU Coulomb gauge fixing failed: %s\n",
            gfix_last_error());
    return 0;
  }
  printf("[GF] Initial Tlink :: %1.15f || Slink :: %1.15f \n"
         "[GF] Plaquette :: %1.15f \n", dg0[1], dg0[0], obs0[2]);
  scatter(L, buf.p, V);
  printf("[GF] Tuning :: %f || Iterations :: %zu ||\n[GF] Final Tlink :: %1.15f "
         "|| Slink :: %1.15f \n[GF] Plaquette :: %1.15f \n",
         Latt.gf_alpha, r.iters, dg[1], dg[0], obs[2]);
  return r.iters;
}

void FOURIER_ACCELERATE2(struct fftw_stuff *FFTW) {
  // one time slice: 4 fields of Lcu complex numbers (CFACG.c:69-88)
  glu_fftw_stuff *F = reinterpret_cast<glu_fftw_stuff *>(FFTW);
  size_t d[4];
  dims_of(d);
  const size_t lcu = d[0] * d[1] * d[2];
  std::vector<double> f(lcu * 8);
  for (int k = 0; k < 4; k++)
    memcpy(f.data() + (size_t)k * lcu * 2, F->in[k], lcu * 2 * sizeof(double));
  if (gfix_fourier_accelerate(f.data(), d, 3) != 0) {
    fprintf(stderr, "[GF] GPU Fourier acceleration failed: %s\n",
            gfix_last_error());
    return;
  }
  for (int k = 0; k < 4; k++)
    memcpy(F->in[k], f.data() + (size_t)k * lcu * 2, lcu * 2 * sizeof(double));
}

}  // extern "C"

extern "C" {

/* GLU's momentum-space measurements (src/Cuts/cuts.c:110-184) for CUTTYPE =
 * GLUON_PROPS, EXCEPTIONAL and FIELDS: the output file is written to the
 * working directory under output_str_struct's name (GLU's default build),
 * configuration number Latt.flow.  GLU leaves the transformed Lie fields in
 * A; here A is left unchanged.  Other modes return GLU_FAILURE (-1). */
int cuts_struct(struct site *lat, const struct cut_info CUTINFO) {
  glu_site *A = reinterpret_cast<glu_site *>(lat);
  size_t d[4];
  dims_of(d);
  const size_t V = volume();
  gfix_cut_info ci;
  ci.dir = CUTINFO.dir;
  ci.type = CUTINFO.type;
  ci.max_mom = CUTINFO.max_mom;
  ci.definition = CUTINFO.definition;
  ci.angle = CUTINFO.angle;
  ci.cyl_width = CUTINFO.cyl_width;
  Buf buf(V * 72);
  if (!buf.p) {
    fprintf(stderr, "[CUTS] allocation of temporaries failed\n");
    return -1;
  }
  gather(A, buf.p, V);
  double err = 0.0;
  char path[1024];
  if (gfix_cuts_write(buf.p, d, &ci, "./", Latt.flow, &err, path, sizeof path) != 0) {
    fprintf(stderr, "[CUTS] %s\n", gfix_cuts_error());
    return -1;
  }
  fprintf(stdout, "\n[CUTS] P-Space gauge fixing error :: %1.5e \n\n", err);
  fprintf(stdout, "[CUTS] Writing finished...\n[CUTS] Outputting to %s\n", path);
  return 0;
}

}  // extern "C"
