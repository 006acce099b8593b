// GLU's gauge-fixing entry points on top of the flat gfix_* interface.
//
// The caller is GLU (or a program built like it): `lat` is GLU's AoS
// lattice, the lattice shape and GF_TUNE are read from GLU's global Latt.
// Each solve gathers the links chunk by chunk into pinned memory on their
// way to the device, runs the GPU solve, scatters them back the same way,
// and follows GLU's return conventions.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/glu_gfix.h"
#include "drop_in.h"
#include "glu_compat.h"

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

// --- GLU's site lattice to and from the device ---------------------------

constexpr size_t kSiteDoubles = 72;       // 4 links x 9 complex numbers
constexpr size_t kChunkSites = 1u << 16;  // 36 MB of links per chunk
constexpr int kSlots = 3;

// A ring of pinned chunks for the whole process: the gather of chunk k+1
// from GLU's per-link allocations overlaps the copy of chunk k to the
// device, and the scatter of chunk k the copy of chunk k+1 back, so no
// pinned buffer of a whole lattice (1.2 GB at 32^3x64, which takes 0.5-0.9 s
// to pin) is made.  Left to the process's exit, like the engines.
struct Ring {
  std::mutex m;  // one transfer at a time
  double *slot[kSlots] = {};
  cudaEvent_t done[kSlots] = {};
  bool ready = false;
  int init() {
    std::lock_guard<std::mutex> lk(m);
    if (ready) return 0;
    for (int i = 0; i < kSlots; i++) {
      cudaError_t e = cudaSuccess;
      if (!slot[i])
        e = cudaMallocHost(&slot[i], kChunkSites * kSiteDoubles * sizeof(double));
      if (e == cudaSuccess && !done[i])
        e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return gfix::cuda_failure("pinned staging chunks", e);
    }
    ready = true;
    return 0;
  }
};

Ring &ring() {
  static Ring *r = new Ring;  // never destroyed: see Warmup
  return *r;
}

// lat[i].O[mu] (separate 144-byte allocations) <-> chunks of double[n][4][18]
struct SiteLinks final : gfix::LinkIO {
  glu_site *lat;
  explicit SiteLinks(glu_site *l) : lat(l) {}
  int to_device(double *d_aos, size_t V, cudaStream_t s) override {
    Ring &R = ring();
    std::lock_guard<std::mutex> lk(R.m);
    for (size_t i0 = 0, k = 0; i0 < V; i0 += kChunkSites, k++) {
      const int j = (int)(k % kSlots);
      const size_t n = std::min(kChunkSites, V - i0);
      // the slot's previous copy has left it
      cudaError_t e = cudaEventSynchronize(R.done[j]);
      if (e != cudaSuccess) return gfix::cuda_failure("staging copy", e);
      gather(lat + i0, R.slot[j], n);
      e = cudaMemcpyAsync(d_aos + i0 * kSiteDoubles, R.slot[j],
                          n * kSiteDoubles * sizeof(double), cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaEventRecord(R.done[j], s);
      if (e != cudaSuccess) return gfix::cuda_failure("staging copy", e);
    }
    return 0;
  }
  int to_host(const double *d_aos, size_t V, cudaStream_t s) override {
    Ring &R = ring();
    std::lock_guard<std::mutex> lk(R.m);
    const size_t nch = (V + kChunkSites - 1) / kChunkSites;
    auto issue = [&](size_t k) {
      const int j = (int)(k % kSlots);
      const size_t i0 = k * kChunkSites, n = std::min(kChunkSites, V - i0);
      cudaError_t e = cudaMemcpyAsync(R.slot[j], d_aos + i0 * kSiteDoubles,
                                      n * kSiteDoubles * sizeof(double),
                                      cudaMemcpyDeviceToHost, s);
      return e == cudaSuccess ? cudaEventRecord(R.done[j], s) : e;
    };
    for (size_t k = 0; k < nch && k < (size_t)kSlots; k++)
      if (cudaError_t e = issue(k)) return gfix::cuda_failure("return copy", e);
    for (size_t k = 0; k < nch; k++) {
      const int j = (int)(k % kSlots);
      const size_t i0 = k * kChunkSites;
      if (cudaError_t e = cudaEventSynchronize(R.done[j]))
        return gfix::cuda_failure("return copy", e);
      scatter(lat + i0, R.slot[j], std::min(kChunkSites, V - i0));
      if (k + kSlots < nch)
        if (cudaError_t e = issue(k + kSlots)) return gfix::cuda_failure("return copy", e);
    }
    return 0;
  }
};

// Inside a GLU program the device context is created, and the ring
// allocated, on a thread started when the library is loaded, while the
// program starts up, reads and checks its configuration (creating the
// context takes up to 1.9 s on a B200); every entry point waits for that
// thread before its own first CUDA call.  The program's CUDA modules --
// this library's -- are loaded with the context (CUDA_MODULE_LOADING=EAGER
// unless the environment sets it), not at each kernel's first launch
// inside the call: at 32^3x64 Landau() then took 0.82-0.85 s (FP64) and
// 0.56-0.64 s (mixed) inside GLU's program in most runs, against 0.79 and
// 0.53 s for the flat driver on links already in pinned memory with its
// workspaces warm.  A program
// is GLU's when its own definition of Latt overrides the library's weak
// one.  GLU_GFIX_PREINIT=0 turns all this off.  The thread is detached and
// its state never destroyed, so that a program which exits without
// calling in does not wait for it.
struct Warmup {
  std::mutex m;
  std::condition_variable cv;
  bool running = false;
  void start() {
    running = true;
    std::thread([this] {
      if (cudaFree(nullptr) == cudaSuccess) ring().init();
      cudaGetLastError();  // a failure is met again, and reported, by the call
      std::lock_guard<std::mutex> lk(m);
      running = false;
      cv.notify_all();
    }).detach();
  }
  void wait() {
    std::unique_lock<std::mutex> lk(m);
    cv.wait(lk, [this] { return !running; });
  }
};

Warmup &warmup() {
  static Warmup *w = new Warmup;
  return *w;
}

bool in_glu_program() {
  Dl_info latt{}, self{};
  if (!dladdr((const void *)&Latt, &latt) || !dladdr((const void *)&in_glu_program, &self))
    return false;
  return latt.dli_fbase != self.dli_fbase;
}

__attribute__((constructor)) void preinit_in_glu_program() {
  const char *s = getenv("GLU_GFIX_PREINIT");
  if ((s && atoi(s) == 0) || !in_glu_program()) return;
  setenv("CUDA_MODULE_LOADING", "EAGER", 0);  // before the runtime starts
  warmup().start();
}

// the device, then the ring; 0, or -1 with the reason printed under tag
int ready_to_stage(const char *tag) {
  warmup().wait();
  if (ring().init() == 0) return 0;
  fprintf(stderr, "[%s] allocation of the GPU staging chunks failed: %s\n", tag,
          gfix_last_error());
  return -1;
}

// GLU_GFIX_TIMING=1: one line per GLU-named solve with the wall time of
// each of its phases -- waiting for the device, the staging chunks, the
// workspaces ("engine"), the links' way to the device with their gather,
// the solve, the reunitarisation and diagnostics ("post"), the way back
// with the scatter -- for a program whose own timer covers the whole call
struct Phases {
  bool on = false;
  double last = 0.0;
  char line[320] = {0};
  size_t len = 0;
  static double now() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
  }
  static void mark_cb(void *self, const char *phase) {
    static_cast<Phases *>(self)->mark(phase);
  }
  Phases() {
    const char *s = getenv("GLU_GFIX_TIMING");
    on = s && atoi(s) != 0;
    last = now();
    if (on) gfix::set_phase_mark(mark_cb, this);
  }
  ~Phases() {
    if (on) gfix::set_phase_mark(nullptr, nullptr);
  }
  void mark(const char *name) {
    if (!on) return;
    const double t = now();
    if (len < sizeof line)
      len += snprintf(line + len, sizeof line - len, " || %s %.3e s", name, t - last);
    last = t;
  }
  void print() const {
    if (on) printf("[GF] GPU timing%s\n", line);
  }
};

size_t landau_fa(glu_site *lat, double *th, double acc, size_t max_iters,
                 int algo) {
  size_t d[4];
  dims_of(d);
  if (ready_to_stage("FACG")) return 0;
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
  SiteLinks io(lat);
  if (gfix::landau_io(io, d, &p, &r) != 0) {
    fprintf(stderr, "[GF] GPU gauge fixing failed: %s\n", gfix_last_error());
    return 0;
  }
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
  warmup().wait();
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
  Phases ph;
  warmup().wait();
  ph.mark("device");
  if (ready_to_stage("GF")) return kGluFailure;
  ph.mark("chunks");
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
  SiteLinks io(L);
  gfix::set_restart_log(true);
  // the links of the last attempt go back to the caller either way
  const int rc = gfix::landau_driver_io(io, d, &p, &r, obs, dg);
  gfix::set_restart_log(false);
  if (rc != 0) {
    fprintf(stderr, "[GF] GPU gauge fixing failed: %s\n", gfix_last_error());
    return kGluFailure;
  }
  ph.print();
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
  if (ready_to_stage("CG")) return 0;
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
  SiteLinks io(L);
  if (gfix::coulomb_io(io, d, &p, &r, nullptr, nullptr) != 0) {
    fprintf(stderr, "[CG] GPU Coulomb gauge fixing failed: %s\n",
            gfix_last_error());
    return 0;
  }
  return r.iters;
}

size_t Coulomb(struct site *lat, const double accuracy, const size_t iter) {
  glu_site *L = reinterpret_cast<glu_site *>(lat);
  size_t d[4];
  dims_of(d);
  Phases ph;
  warmup().wait();
  ph.mark("device");
  if (ready_to_stage("CG")) return 0;
  ph.mark("chunks");
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
  SiteLinks io(L);
  if (gfix::coulomb_driver_io(io, d, &p, &r, obs0, dg0, obs, dg) != 0) {
    fprintf(stderr, "[CG] GPU Coulomb gauge fixing failed: %s\n",
            gfix_last_error());
    return 0;
  }
  ph.print();
  printf("[GF] Initial Tlink :: %1.15f || Slink :: %1.15f \n"
         "[GF] Plaquette :: %1.15f \n", dg0[1], dg0[0], obs0[2]);
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
  warmup().wait();
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
  std::unique_ptr<double[]> buf(new (std::nothrow) double[V * kSiteDoubles]);
  if (!buf) {
    fprintf(stderr, "[CUTS] allocation of temporaries failed\n");
    return -1;
  }
  gather(A, buf.get(), V);
  warmup().wait();
  double err = 0.0;
  char path[1024];
  if (gfix_cuts_write(buf.get(), d, &ci, "./", Latt.flow, &err, path, sizeof path) != 0) {
    fprintf(stderr, "[CUTS] %s\n", gfix_cuts_error());
    return -1;
  }
  fprintf(stdout, "\n[CUTS] P-Space gauge fixing error :: %1.5e \n\n", err);
  fprintf(stdout, "[CUTS] Writing finished...\n[CUTS] Outputting to %s\n", path);
  return 0;
}

}  // extern "C"
