// Host engine and C ABI of the B200 Fourier-accelerated gauge fixing.
//
// An Engine<R> owns the device workspace of one lattice shape in working
// precision R: SoA links, the in/in_old and sn ping-pong fields, partial
// sums, twiddle and cos tables, a device-side control block (DevState) and
// the CUDA graphs of one solver iteration.  The solver loops replay a graph
// and only read the control block back every few iterations; all of GLU's
// scalar control flow (theta, beta, alpha*, stop tests) runs on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/glu_gfix.h"
#include "coulomb.cuh"
#include "drop_in.h"
#include "extra_kernels.cuh"
#include "kernels.cuh"

namespace gfix {

static thread_local std::string g_err = "";
static std::atomic<unsigned long long> g_launches{0};

static int fail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return -1;
}

#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess)                                              \
      return fail("%s:%d %s: %s", __FILE__, __LINE__, #call,           \
                  cudaGetErrorString(e_));                              \
  } while (0)

#define LAUNCHED(n) g_launches.fetch_add((n), std::memory_order_relaxed)

// kernels launched by the other translation units of the library
void count_launches(unsigned long long n) { LAUNCHED(n); }

constexpr size_t kSentinel = 123456789;
constexpr size_t kGluFailure = (size_t)-1;  // GLU_FAILURE returned as size_t

// FFT plans: 0 = the default plan per shape (bit-reproducible runs), 1 =
// autotuned per shape at first use (gfix_fft_tuning, GLU_GFIX_FFT_TUNE=1)
static int g_fft_tune = -1;
static int fft_tuning() {
  if (g_fft_tune < 0) {
    const char *e = getenv("GLU_GFIX_FFT_TUNE");
    g_fft_tune = (e && atoi(e) != 0) ? 1 : 0;
  }
  return g_fft_tune;
}

// compile-time specialised FFT passes for the common extents; nullptr
// where the generic passes serve
template <typename R>
using XyFn = void (*)(Ctx<R>, int, int);
template <typename R>
using ZtFn = void (*)(Ctx<R>);

template <typename R>
static XyFn<R> ct_xy(int lx, int ly) {
#define GFIX_XY(n) \
  if (lx == n && ly == n) return k_fft_xy_ct<R, n, n>;
  GFIX_XY(4) GFIX_XY(8) GFIX_XY(16) GFIX_XY(24) GFIX_XY(32) GFIX_XY(48)
  GFIX_XY(64)
#undef GFIX_XY
  return nullptr;
}

template <typename R>
static ZtFn<R> ct_zt(int lz, int lt, int b) {
#define GFIX_ZT(z, t, bb) \
  if (lz == z && lt == t && b == bb) return k_fft_zt_ct<R, z, t, bb>;
  GFIX_ZT(4, 4, 2) GFIX_ZT(4, 8, 2) GFIX_ZT(8, 8, 2) GFIX_ZT(8, 16, 2)
  GFIX_ZT(16, 16, 2) GFIX_ZT(16, 32, 2) GFIX_ZT(24, 48, 2)
  GFIX_ZT(32, 32, 2) GFIX_ZT(32, 64, 2) GFIX_ZT(48, 96, 2)
  GFIX_ZT(32, 64, 1) GFIX_ZT(32, 64, 4) GFIX_ZT(48, 96, 1) GFIX_ZT(16, 32, 4)
  GFIX_ZT(4, 1, 8) GFIX_ZT(8, 1, 8) GFIX_ZT(16, 1, 8) GFIX_ZT(24, 1, 8)
  GFIX_ZT(32, 1, 8) GFIX_ZT(48, 1, 8) GFIX_ZT(64, 1, 8)
  GFIX_ZT(8, 1, 16) GFIX_ZT(16, 1, 16) GFIX_ZT(24, 1, 16) GFIX_ZT(32, 1, 16)
  GFIX_ZT(48, 1, 16) GFIX_ZT(64, 1, 16) GFIX_ZT(32, 1, 32) GFIX_ZT(64, 1, 32)
#undef GFIX_ZT
  return nullptr;
}

struct Params {
  double gf_alpha = 0.08, acc = 1e-14;
  size_t max_iters = 1000;
  int algo = GFIX_CG, sd_fixed = 0;
  double *traj_theta = nullptr, *traj_func = nullptr;
  size_t traj_cap = 0;
  // stall rule (DevState), set for mixed-precision FP32 phases only
  long long stall_window = 0;
  double stall_floor = 0.0, blowup = 0.0;
};

// The FP32 phase of a mixed-precision solve hands over to FP64 at
// switch_theta, or earlier when it stops making progress: on thermalised
// fields theta crosses long plateaus on which FP32 arithmetic can lose the
// ground it had gained (theta jumping by orders of magnitude), so once the
// best theta is below 1e-4 the phase ends after 15 iterations without a
// 10% improvement or on a jump above 30x the best (the window of the best
// mean over four beta 6.0 heatbath configurations of 32^3x64 among 15, 25
// and 40; on smoothly converging inputs the rule never fires).
// GLU_GFIX_STALL="window,floor,blowup" overrides it ("0": switch at
// switch_theta only).  CG only: steepest descent (FASD) converges slowly but
// steadily in FP32 -- its FP32 steps track the FP64 ones -- and the rule
// would only cut its FP32 phase short (measured on beta 5.9 / 6.0
// configurations: 73 ms without the rule, 111 ms with it, 116 ms in FP64).
static void stall_rule(Params &p) {
  if (p.algo != GFIX_CG) return;
  p.stall_window = 15;
  p.stall_floor = 1e-4;
  p.blowup = 30.0;
  if (const char *e = getenv("GLU_GFIX_STALL")) {
    long long w = 0;
    double f = 0.0, b = 0.0;
    const int n = sscanf(e, "%lld,%lf,%lf", &w, &f, &b);
    p.stall_window = n >= 1 ? w : 0;
    if (n >= 2) p.stall_floor = f;
    if (n >= 3) p.blowup = b;
  }
}

// R: links and their arithmetic; F: the su(3) fields and the FFT (F = R,
// or float under FP64 links in the FP64 phase of a mixed-precision solve)
template <typename R, typename F = R>
class Engine {
 public:
  size_t dims[4] = {0, 0, 0, 0};
  int V = 0;
  Ctx<R, F> c{};
  cudaStream_t s = nullptr;
  DevState *d_st = nullptr, *h_st = nullptr;
  double *d_part = nullptr, *d_cs = nullptr, *d_traj = nullptr;
  cx<F> *d_tw = nullptr, *d_F = nullptr;
  cx<R> *d_U = nullptr, *d_G = nullptr;
  double *d_aos = nullptr;  // AoS FP64 staging (only FP64 engines)
  cx<R> *d_best = nullptr;  // luxury copies: the kept copy's links
  // sequences (landau_sequence): a second AoS buffer and a copy stream
  double *d_aos2 = nullptr;
  cudaStream_t s_copy = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_solved = nullptr;
  size_t traj_alloc = 0;
  int nb_site = 0;
  dim3 g_xy, g_zt;
  size_t sm_xy = 0, sm_zt = 0;
  int bd_xy = 256, bd_zt = 256, pt_xy = 8, pt_zt = 8;
  bool odd = false;
  bool coul = false;
  int Lcu = 0;
  XyFn<F> xy_ct = nullptr;
  ZtFn<F> zt_ct = nullptr;
  cudaGraphExec_t gx_cg = nullptr, gx_sd = nullptr;
  cudaGraph_t gr_cg = nullptr, gr_sd = nullptr;  // the same, uninstantiated
  int gx_sd_fixed = -1;
  bool primed = false;
  bool graph_ok = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  ~Engine() { release(); }

  void release() {
    if (gx_cg) cudaGraphExecDestroy(gx_cg);
    if (gx_sd) cudaGraphExecDestroy(gx_sd);
    if (gx_coul) cudaGraphExecDestroy(gx_coul);
    if (gr_cg) cudaGraphDestroy(gr_cg);
    if (gr_sd) cudaGraphDestroy(gr_sd);
    gx_cg = gx_sd = gx_coul = nullptr;
    gr_cg = gr_sd = nullptr;
    cudaFree(d_cst);
    cudaFreeHost(h_cst);
    cudaFree(d_sl);
    cudaFreeHost(h_sl);
    cudaFree(d_ctraj);
    cudaFree(d_cmask);
    d_cmask = nullptr;
    d_cst = nullptr;
    d_sl = nullptr;
    cudaFree(d_st);
    cudaFreeHost(h_st);
    cudaFree(d_part);
    cudaFree(d_cs);
    cudaFree(d_traj);
    cudaFree(d_tw);
    cudaFree(d_U);
    cudaFree(d_F);
    cudaFree(d_G);
    cudaFree(d_aos);
    cudaFree(d_best);
    d_best = nullptr;
    cudaFree(d_aos2);
    d_aos2 = nullptr;
    for (cudaEvent_t &ev : ev_in)
      if (ev) cudaEventDestroy(ev), ev = nullptr;
    if (ev_solved) cudaEventDestroy(ev_solved), ev_solved = nullptr;
    if (s_copy) cudaStreamDestroy(s_copy), s_copy = nullptr;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
    d_st = nullptr;
    h_st = nullptr;
    s = nullptr;
  }

  int init(const size_t *d, bool with_G, bool with_staging,
           bool coulomb = false) {
    coul = coulomb;
    for (int i = 0; i < 4; i++) dims[i] = d[i];
    const size_t Vs = d[0] * d[1] * d[2] * d[3];
    if (Vs == 0 || Vs > (size_t)INT32_MAX / 4)
      return fail("lattice volume %zu outside 1..2^29", Vs);
    V = (int)Vs;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    for (int i = 0; i < 4; i++) {
      c.L[i] = (int)d[i];
      if (factorize(c.L[i], c.ax[i]) != 0)
        return fail("extent %d has a prime factor above %d", c.L[i], kMaxRadix);
    }
    c.V = V;
    Lcu = (int)(d[0] * d[1] * d[2]);
    c.ndim = coul ? 3 : 4;
    // MAX_LANDAU = 4 ND / V, MAX_COULOMB = 4 (ND - 1) / LCU
    // (GLU_definitions.h:414, 420)
    c.maxp = coul ? 4.0 * 3 / (double)Lcu : 4.0 * 4 / (double)V;
    // twiddle pool: one table per axis
    std::vector<cx<F>> tw;
    for (int a = 0; a < 4; a++) {
      c.ax[a].tw_off = (int)tw.size();
      const int n = c.L[a];
      for (int k = 0; k < n; k++) {
        const double ang = 6.283185307179586476925286766559 * k / n;
        tw.push_back(mk<F>((F)std::cos(ang), (F)(-std::sin(ang))));
      }
    }
    CK(cudaMalloc(&d_tw, tw.size() * sizeof(cx<F>)));
    CK(cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(cx<F>),
                  cudaMemcpyHostToDevice));
    c.tw = d_tw;
    // cos tables as GLU evaluates them: cos(n * (TWOPI / L)) (init.c:66,
    // geometry.c:176)
    const int ld = *std::max_element(c.L, c.L + 4);
    std::vector<double> cs(4 * (size_t)ld, 0.0);
    for (int a = 0; a < 4; a++) {
      const double twd = 6.283185307179586 / (double)c.L[a];
      for (int n = 0; n < c.L[a]; n++) cs[a * ld + n] = std::cos(n * twd);
    }
    CK(cudaMalloc(&d_cs, cs.size() * sizeof(double)));
    CK(cudaMemcpy(d_cs, cs.data(), cs.size() * sizeof(double),
                  cudaMemcpyHostToDevice));
    c.cs = d_cs;
    c.cs_ld = ld;
    // tiles
    c.xy_pitch = c.L[0] + 1;
    // x columns per zt tile: Landau's (z, t) tiles take 4 where a
    // compile-time pass for them exists (the autotuner's pick on 16^3x32
    // and 32^3x64), else 2 (32-byte rows in FP64); Coulomb tiles hold one
    // slice's z pencils only and take 16
    odd = false;
    for (int a = 0; a < 4; a++)
      for (int k = 0; k < c.ax[a].nstages; k++)
        odd |= (c.ax[a].st[k].r == 5 || c.ax[a].st[k].r == 7);
    const int nt = coul ? 1 : c.L[3];
    int want_b = coul ? 16 : 2;
    if (!coul && !odd && c.L[0] % 4 == 0 && ct_zt<F>(c.L[2], nt, 4) != nullptr &&
        zt_smem(4) <= 200u * 1024u)
      want_b = 4;
    c.zt_b = 1;
    for (int b = want_b; b >= 1; b--)
      if (c.L[0] % b == 0) {
        c.zt_b = b;
        break;
      }
    // a compile-time pass takes the tile as chosen while its shared memory
    // fits (tiles up to 16384 elements); the generic passes hold one
    // element per thread and stage for 8 (16) elements: tiles up to 8192
    const bool ct_tile = !odd && ct_zt<F>(c.L[2], nt, c.zt_b) != nullptr &&
                         zt_smem(c.zt_b) <= 200u * 1024u;
    if (!ct_tile) {
      while (c.zt_b > 1 && (size_t)c.zt_b * c.L[2] * nt > 4096u) c.zt_b /= 2;
      while (c.zt_b > 1 && c.L[0] % c.zt_b) c.zt_b /= 2;
    }
    if ((size_t)c.L[0] * c.L[1] > 8192)
      return fail("FFT xy tile of %d elements exceeds 8192", c.L[0] * c.L[1]);
    // tile (padded) plus the twiddle tables of its two axes
    sm_xy = ((size_t)c.xy_pitch * c.L[1] + c.L[0] + c.L[1]) * sizeof(cx<F>);
    // the dynamic shared-memory limit is an attribute of the function, not
    // of a launch: raise it once to the largest tile any engine can use
    if (set_smem_limits()) return -1;
    // default plan (FFTW's ESTIMATE, so to speak): compile-time passes where
    // the extents have one, largest radices first
    if (apply_xy(true, 0) && apply_xy(false, 0))
      return fail("no xy FFT pass for %d x %d", c.L[0], c.L[1]);
    if (apply_zt(c.zt_b, ct_tile, 0) && apply_zt(c.zt_b, false, 0))
      return fail("FFT tile of %zu elements exceeds 8192",
                  (size_t)c.zt_b * c.L[2] * nt);
    g_xy = dim3(V / (c.L[0] * c.L[1]), 4);
    nb_site = (V + kSiteThreads - 1) / kSiteThreads;
    const size_t nparts =
        std::max<size_t>((size_t)nb_site, (size_t)g_xy.x * g_xy.y) + 1024;
    CK(cudaMalloc(&d_part, nparts * 2 * sizeof(double)));
    c.part = d_part;
    CK(cudaMalloc(&d_st, sizeof(DevState)));
    CK(cudaMallocHost(&h_st, sizeof(DevState)));
    memset(h_st, 0, sizeof(DevState));
    c.st = d_st;
    CK(cudaMalloc(&d_U, (size_t)V * 4 * kLinkCx * sizeof(cx<R>)));
    CK(cudaMalloc(&d_F, (size_t)V * 16 * sizeof(cx<F>)));
    c.U = d_U;
    c.fb[0] = d_F;
    c.fb[1] = d_F + (size_t)4 * V;
    c.sb[0] = d_F + (size_t)8 * V;
    c.sb[1] = d_F + (size_t)12 * V;
    if (with_G) CK(cudaMalloc(&d_G, (size_t)V * 9 * sizeof(cx<R>)));
    c.G = d_G;
    if (with_staging) CK(cudaMalloc(&d_aos, (size_t)V * 36 * sizeof(double2)));
    if (fft_tuning() && tune_fft()) return -1;
    return 0;
  }

  // --- FFT plans ------------------------------------------------------
  size_t zt_smem(int b) const {
    return coul ? ((size_t)b * c.L[2] + c.L[2]) * sizeof(cx<F>)
                : ((size_t)(b * c.L[2] + std::max(1, zt_pad(b))) * c.L[3] +
                   c.L[2] + c.L[3]) * sizeof(cx<F>);
  }
  static size_t threads_for(size_t n, int pt) {
    size_t t = (n + pt - 1) / pt;
    return std::max<size_t>(128, (t + 31) / 32 * 32);
  }
  // the xy pass: compile-time (use_ct) or generic with radix order `order`;
  // -1 where that pass does not exist for these extents
  int apply_xy(bool use_ct, int order) {
    for (int a = 0; a < 2; a++)
      if (factorize(c.L[a], c.ax[a], order)) return -1;
    const size_t n = (size_t)c.L[0] * c.L[1];
    if (use_ct) {
      XyFn<F> fn = odd ? nullptr : ct_xy<F>(c.L[0], c.L[1]);
      if (!fn) return -1;
      xy_ct = fn;
      bd_xy = ct_threads((int)n);
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sm_xy));
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared));
    } else {
      xy_ct = nullptr;
      pt_xy = (n <= 4096u && !odd) ? 8 : 16;
      bd_xy = (int)threads_for(n, pt_xy);
    }
    xy_plan = use_ct ? -1 : order;
    return 0;
  }
  // the z(,t) pass with tiles of b x columns
  int apply_zt(int b, bool use_ct, int order) {
    const int nt = coul ? 1 : c.L[3];
    if (b < 1 || c.L[0] % b) return -1;
    for (int a = 2; a < 4; a++)
      if (factorize(c.L[a], c.ax[a], order)) return -1;
    const size_t n = (size_t)b * c.L[2] * nt;
    if (use_ct) {
      ZtFn<F> fn = odd ? nullptr : ct_zt<F>(c.L[2], nt, b);
      if (!fn || zt_smem(b) > 200u * 1024u) return -1;
      zt_ct = fn;
      bd_zt = zt_threads<F>((int)n);
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)zt_smem(b)));
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared));
    } else {
      if (n > 8192) return -1;
      zt_ct = nullptr;
      pt_zt = (n <= 4096u && !odd) ? 8 : 16;
      bd_zt = (int)threads_for(n, pt_zt);
    }
    c.zt_b = b;
    sm_zt = zt_smem(b);
    g_zt = dim3((c.L[0] / b) * c.L[1] * (coul ? c.L[3] : 1), 4);
    zt_plan = use_ct ? -1 : order;
    return 0;
  }
  int xy_plan = -1, zt_plan = -1;  // -1 compile-time pass, else radix order

  // FFTW's MEASURE, so to speak: time every available xy and zt pass once
  // for these extents (compile-time or generic, each radix order; every zt
  // tile width dividing Lx) and keep the fastest.  One plan per shape and
  // precision and process; plans change rounding, not results beyond it.
  struct TunedPlan {
    bool xy_ct;
    int xy_order, zt_b;
    bool zt_ct;
    int zt_order;
    float xy_ms, zt_ms;
  };
  static std::map<std::tuple<int, int, int, int, bool>, TunedPlan> &tuned() {
    static std::map<std::tuple<int, int, int, int, bool>, TunedPlan> m;
    return m;
  }
  int time_pass(bool xy, float *ms) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int k = 0; k < 2; k++) xy ? fft_xy(0, 0) : fft_zt();
    CK(cudaEventRecord(a, s));
    for (int k = 0; k < 5; k++) xy ? fft_xy(0, 0) : fft_zt();
    CK(cudaEventRecord(b, s));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(ms, a, b));
    *ms /= 5.f;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  int tune_fft() {
    const auto key = std::make_tuple(c.L[0], c.L[1], c.L[2], c.L[3], coul);
    auto it = tuned().find(key);
    TunedPlan P;
    if (it == tuned().end()) {
      Params p;
      if (reset(p)) return -1;
      CK(cudaMemsetAsync(d_F, 0, (size_t)V * 16 * sizeof(cx<F>), s));
      float best = 1e30f, t = 0.f;
      P = TunedPlan{xy_ct != nullptr, xy_plan < 0 ? 0 : xy_plan, c.zt_b,
                    zt_ct != nullptr, zt_plan < 0 ? 0 : zt_plan, 0.f, 0.f};
      for (int ct = 1; ct >= 0; ct--)
        for (int o = 0; o < (ct ? 1 : kRadixOrders); o++) {
          if (apply_xy(ct != 0, o)) continue;
          if (time_pass(true, &t)) return fail("FFT autotuning failed");
          if (t < best) {
            best = t;
            P.xy_ct = ct != 0;
            P.xy_order = o;
            P.xy_ms = t;
          }
        }
      best = 1e30f;
      for (int b = 1; b <= 32; b *= 2)
        for (int ct = 1; ct >= 0; ct--)
          for (int o = 0; o < (ct ? 1 : kRadixOrders); o++) {
            if (apply_zt(b, ct != 0, o)) continue;
            if (time_pass(false, &t)) return fail("FFT autotuning failed");
            if (t < best) {
              best = t;
              P.zt_b = b;
              P.zt_ct = ct != 0;
              P.zt_order = o;
              P.zt_ms = t;
            }
          }
      tuned()[key] = P;
    } else {
      P = it->second;
    }
    if (apply_xy(P.xy_ct, P.xy_order) || apply_zt(P.zt_b, P.zt_ct, P.zt_order))
      return fail("tuned FFT plan not applicable");
    return 0;
  }

  int ensure_traj(size_t cap) {
    if (cap <= traj_alloc) return 0;
    cudaFree(d_traj);
    d_traj = nullptr;
    traj_alloc = 0;
    CK(cudaMalloc(&d_traj, 2 * cap * sizeof(double)));
    traj_alloc = cap;
    return 0;
  }

  // --- launch sequences ------------------------------------------------
  void scalar(int op, int nv) {
    k_scalar<<<1, kScalarThreads, 0, s>>>(d_st, d_part, op, nv, (double)V);
    LAUNCHED(1);
  }
  void theta(int op) {
    k_deriv<R, F><<<nb_site, kSiteThreads, 0, s>>>(c);
    LAUNCHED(1);
    scalar(op, 2);
  }
  static int set_smem_limits() {
    static bool done = false;
    if (done) return 0;
    const int lim = (8192 + 8192 / 8 + 1024) * (int)sizeof(cx<F>);
    const void *fns[] = {
        (const void *)k_fft_xy<F, 8, false>, (const void *)k_fft_xy<F, 16, false>,
        (const void *)k_fft_xy<F, 16, true>, (const void *)k_fft_zt<F, 8, false>,
        (const void *)k_fft_zt<F, 16, false>, (const void *)k_fft_zt<F, 16, true>};
    for (const void *f : fns) {
      CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
      CK(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared));
    }
    done = true;
    return 0;
  }
  // the context the FFT passes and field-only kernels see: the fields'
  // type throughout (they touch neither links nor G)
  Ctx<F> cf() const {
    if constexpr (std::is_same<R, F>::value) {
      return c;
    } else {
      Ctx<F> v;
      v.U = nullptr;
      v.G = nullptr;
      v.fb[0] = c.fb[0];
      v.fb[1] = c.fb[1];
      v.sb[0] = c.sb[0];
      v.sb[1] = c.sb[1];
      v.st = c.st;
      v.part = c.part;
      v.tw = c.tw;
      v.cs = c.cs;
      v.cs_ld = c.cs_ld;
      for (int i = 0; i < 4; i++) {
        v.L[i] = c.L[i];
        v.ax[i] = c.ax[i];
      }
      v.V = c.V;
      v.ndim = c.ndim;
      v.zt_b = c.zt_b;
      v.xy_pitch = c.xy_pitch;
      v.maxp = c.maxp;
      v.skip = c.skip;
      return v;
    }
  }
  void fft_xy(int bwd, int prsum) {
    const Ctx<F> v = cf();
    if (xy_ct)
      xy_ct<<<g_xy, bd_xy, sm_xy, s>>>(v, bwd, prsum);
    else if (odd)
      k_fft_xy<F, 16, true><<<g_xy, bd_xy, sm_xy, s>>>(v, bwd, prsum);
    else if (pt_xy == 8)
      k_fft_xy<F, 8, false><<<g_xy, bd_xy, sm_xy, s>>>(v, bwd, prsum);
    else
      k_fft_xy<F, 16, false><<<g_xy, bd_xy, sm_xy, s>>>(v, bwd, prsum);
    LAUNCHED(1);
  }
  void fft_zt() {
    const Ctx<F> v = cf();
    if (zt_ct)
      zt_ct<<<g_zt, bd_zt, sm_zt, s>>>(v);
    else if (odd)
      k_fft_zt<F, 16, true><<<g_zt, bd_zt, sm_zt, s>>>(v);
    else if (pt_zt == 8)
      k_fft_zt<F, 8, false><<<g_zt, bd_zt, sm_zt, s>>>(v);
    else
      k_fft_zt<F, 16, false><<<g_zt, bd_zt, sm_zt, s>>>(v);
    LAUNCHED(1);
  }
  // direction + probes: FP64 storage one kernel; FP32 storage the FP32- and
  // the FP64-arithmetic variants, of which the device state picks one
  template <bool DIR>
  void probe() {
    if (sizeof(R) == 8) {
      k_dir_probe<R, DIR, double, F><<<nb_site, kSiteThreads, 0, s>>>(c, SEL_ALWAYS);
    } else {
      k_dir_probe<R, DIR, R, F><<<nb_site, kSiteThreads, 0, s>>>(c, SEL_LOW);
      k_dir_probe<R, DIR, double, F><<<nb_site, kSiteThreads, 0, s>>>(c, SEL_HIGH);
      LAUNCHED(1);
    }
  }
  void fft(bool prsum) {
    fft_xy(0, 0);
    fft_zt();
    fft_xy(1, prsum ? 1 : 0);
  }
  // an SD step (steep_Landau_FA, src/Gfix/FACG.c:181-199); main = one FASD
  // iteration with its stop test
  void sd_step(bool main, bool sd_fixed) {
    theta(main ? OP_THETA_MAIN : OP_THETA_SD);
    fft(false);
    if (sd_fixed) {
      scalar(OP_ALPHA_FIXED, 0);
    } else {
      probe<false>();
      LAUNCHED(1);
      scalar(OP_PROBES, 2);
    }
    k_update<R, false, F><<<nb_site, kSiteThreads, 0, s>>>(c);
    LAUNCHED(1);
    if (main) scalar(OP_END_SD, 0);
  }
  // one CG iteration (src/Gfix/FACG.c:270-334)
  void cg_iter() {
    theta(OP_THETA_MAIN);
    fft(true);
    scalar(OP_PR, 2);
    probe<true>();
    LAUNCHED(1);
    scalar(OP_PROBES, 2);
    k_update<R, true, F><<<nb_site, kSiteThreads, 0, s>>>(c);
    LAUNCHED(1);
    scalar(OP_END_CG, 0);
  }

  // Launch every kernel of the iteration once with the done flag set: each
  // returns at once, but the module loading that CUDA defers to a kernel's
  // first launch happens here and not inside a stream capture.
  int prime() {
    if (primed) return 0;
    k_set_done<<<1, 1, 0, s>>>(d_st, 1);
    cg_iter();
    sd_step(true, false);
    sd_step(true, true);
    k_copy_der<F><<<nb_site, kSiteThreads, 0, s>>>(cf());
    k_set_done<<<1, 1, 0, s>>>(d_st, 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    primed = true;
    return 0;
  }

  int capture(cudaGraphExec_t *out, bool cg, bool sd_fixed) {
    if (prime()) return -1;
    cudaGraph_t g = nullptr;
    CK(cudaGetLastError());
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    const unsigned long long before = g_launches.load();
    if (cg)
      cg_iter();
    else
      sd_step(true, sd_fixed);
    // captured launches run later; they are counted at replay
    g_launches.store(before);
    CK(cudaStreamEndCapture(s, &g));
    CK(cudaGraphInstantiate(out, g, 0));
    // kept for batches, which nest it in a graph over many engines
    cudaGraph_t &keep = cg ? gr_cg : gr_sd;
    if (keep) cudaGraphDestroy(keep);
    keep = g;
    return 0;
  }

  unsigned long long per_iter_launches(bool cg, bool sd_fixed) const {
    // k_deriv + scalar + 3 fft + ...
    // (FP32 storage launches two probe variants)
    const unsigned long long two = sizeof(R) == 4 ? 1 : 0;
    if (cg) return 2 + 3 + 1 + 2 + 1 + 1 + two;
    return 2 + 3 + (sd_fixed ? 1 : 2 + two) + 1 + 1;
  }

  int read_state() {
    CK(cudaMemcpyAsync(h_st, d_st, sizeof(DevState), cudaMemcpyDeviceToHost,
                       s));
    CK(cudaStreamSynchronize(s));
    return 0;
  }

  // replay an iteration (graph, or direct launches when the graph could
  // not be built) until the device says done
  int replay(cudaGraphExec_t gx, bool cg, bool sd_fixed) {
    const unsigned long long per_iter = per_iter_launches(cg, sd_fixed);
    int batch = 2;
    size_t guard = 0;
    for (;;) {
      for (int k = 0; k < batch; k++) {
        if (gx) {
          CK(cudaGraphLaunch(gx, s));
          LAUNCHED(per_iter);
        } else if (cg) {
          cg_iter();
        } else {
          sd_step(true, sd_fixed);
        }
      }
      CK(cudaGetLastError());
      if (read_state()) return -1;
      if (h_st->done) return 0;
      guard += batch;
      if (guard > (size_t)h_st->max_iters + 64)
        return fail("solver did not stop after %zu iterations", guard);
      batch = std::min(batch * 2, 32);
    }
  }

  // build the iteration graph; on failure run without one (graph_ok = 0)
  void ensure_graph(cudaGraphExec_t *gx, bool cg, bool sd_fixed) {
    if (*gx || !graph_ok) return;
    if (capture(gx, cg, sd_fixed)) {
      cudaStreamCaptureStatus st;
      if (cudaStreamIsCapturing(s, &st) == cudaSuccess &&
          st != cudaStreamCaptureStatusNone) {
        cudaGraph_t g;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
      }
      cudaGetLastError();
      *gx = nullptr;
      graph_ok = false;
      fprintf(stderr, "[GF] CUDA graph capture failed (%s); launching the "
              "iteration kernels directly\n", g_err.c_str());
    }
  }

  // state for a new solve
  int reset(const Params &p) {
    if (p.traj_cap && ensure_traj(p.traj_cap)) return -1;
    DevState st;
    memset(&st, 0, sizeof st);
    st.gf_alpha = p.gf_alpha;
    st.acc = p.acc;
    st.max_iters = (long long)p.max_iters;
    st.sd_fixed = p.sd_fixed;
    // GLU's CG_TOL (5e-11) in both phases: with FP64 probe arithmetic the
    // FP32 phase keeps its line search down to the precision switch
    st.cg_tol = 5E-11;
    st.hp_below = 1E-5;
    st.best_tr = 1e300;
    st.stall_window = p.stall_window;
    st.stall_floor = p.stall_floor;
    st.blowup = p.blowup;
    st.traj_cap = p.traj_cap ? (long long)p.traj_cap : 0;
    st.traj_theta = p.traj_cap ? d_traj : nullptr;
    st.traj_func = p.traj_cap ? d_traj + p.traj_cap : nullptr;
    CK(cudaMemcpyAsync(d_st, &st, sizeof st, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return 0;
  }

  int fetch_traj(const Params &p, size_t *len) {
    *len = 0;
    if (!p.traj_cap) return 0;
    if (read_state()) return -1;
    const size_t n = std::min<size_t>((size_t)h_st->traj_len, p.traj_cap);
    if (n) {
      if (p.traj_theta)
        CK(cudaMemcpy(p.traj_theta, d_traj, n * sizeof(double),
                      cudaMemcpyDeviceToHost));
      if (p.traj_func)
        CK(cudaMemcpy(p.traj_func, d_traj + p.traj_cap, n * sizeof(double),
                      cudaMemcpyDeviceToHost));
    }
    *len = n;
    return 0;
  }

  // theta_test_lin of the current links
  int theta_test(double *out) {
    k_begin_run<<<1, 1, 0, s>>>(d_st);
    LAUNCHED(1);
    theta(OP_THETA_TEST);
    if (read_state()) return -1;
    *out = h_st->tr_test;
    return 0;
  }

  // A solve as resumable steps, shared by the single driver (solve) and
  // the batched one (batch_solve):
  //   run_start  reset, theta_test, graph, launch of the first run's head
  //   run_exec   the iteration graph of the run (nullptr: direct launches)
  //   run_after  once the device says done (h_st current): GLU's end of
  //              FACG / FASD, or the head of a continuation run
  // GLU's FACG (src/Gfix/FACG.c:341-391) and FASD (FACG.c:395-446).
  Params run_p;
  bool run_cg = true;
  size_t run_total = 0;
  // warm start of a CG solve (mixed precision): set by the hand-over, which
  // has put in_old into fb[1] and the last direction into sb[0]; run_start
  // then continues the conjugate directions instead of an SD start
  bool warm = false;
  double warm_inold = 0.0;

  void run_head() {
    k_begin_run<<<1, 1, 0, s>>>(d_st);
    LAUNCHED(1);
    if (run_cg) {
      sd_step(false, run_p.sd_fixed != 0);
      k_copy_der<F><<<nb_site, kSiteThreads, 0, s>>>(cf());
      LAUNCHED(1);
      scalar(OP_DER, 1);
    }
  }

  int run_start(const Params &p, bool *fin, size_t *iters, double *th) {
    run_p = p;
    run_cg = p.algo == GFIX_CG;
    run_total = 0;
    *fin = false;
    if (reset(p)) return -1;
    if (theta_test(th)) return -1;
    if (*th < p.acc) {
      *iters = 0;
      *fin = true;
      return 0;
    }
    if (run_cg) {
      ensure_graph(&gx_cg, true, false);
    } else {
      if (gx_sd_fixed != p.sd_fixed) {
        if (gx_sd) cudaGraphExecDestroy(gx_sd);
        gx_sd = nullptr;
        gx_sd_fixed = p.sd_fixed;
      }
      ensure_graph(&gx_sd, false, p.sd_fixed != 0);
    }
    if (warm && run_cg) {
      // (reset left parity = sparity = 0: in_old = fb[1], sn_old = sb[0])
      k_begin_run<<<1, 1, 0, s>>>(d_st);
      LAUNCHED(1);
      CK(cudaMemcpyAsync(&d_st->inold, &warm_inold, sizeof(double),
                         cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
      warm = false;
      return 0;
    }
    warm = false;
    run_head();
    return 0;
  }

  cudaGraphExec_t run_exec() const { return run_cg ? gx_cg : gx_sd; }
  cudaGraph_t run_graph() const { return run_cg ? gr_cg : gr_sd; }

  int run_after(bool *fin, size_t *iters, double *th) {
    *th = h_st->tr;
    const size_t loc = (size_t)h_st->iter;
    *fin = true;
    if (loc >= run_p.max_iters) {
      if (*th < 1E3 * run_p.acc) {  // continuation run
        // (FASD: loc_iters = 0 again, nothing added)
        *fin = false;
        run_head();
        return 0;
      }
      if (run_cg) {
        *iters = kSentinel;
        return 0;
      }
      run_total = kSentinel;
    }
    *iters = run_cg ? loc : run_total + loc;
    return 0;
  }

  int solve(const Params &p, size_t *iters, double *th) {
    bool fin = false;
    if (run_start(p, &fin, iters, th)) return -1;
    while (!fin) {
      if (replay(run_exec(), run_cg, p.sd_fixed != 0)) return -1;
      if (run_after(&fin, iters, th)) return -1;
    }
    return 0;
  }

  // Per-kernel device times of `n` CG iterations launched one by one with
  // events between the launches (no graph).  ms[k] = average duration of
  // one launch of kernel k, bytes[k] = its algorithmic HBM bytes:
  //   0 k_deriv, 1 k_fft_xy fwd, 2 k_fft_zt, 3 k_fft_xy bwd (+PR sums),
  //   4 k_dir_probe, 5 k_update, 6 the four k_scalar launches together
  int profile_cg(const Params &p, int n, double *ms, double *bytes) {
    if (reset(p)) return -1;
    k_begin_run<<<1, 1, 0, s>>>(d_st);
    sd_step(false, p.sd_fixed != 0);
    k_copy_der<F><<<nb_site, kSiteThreads, 0, s>>>(cf());
    scalar(OP_DER, 1);
    LAUNCHED(2);
    std::vector<cudaEvent_t> ev(8);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int it = 0; it < n; it++) {
      CK(cudaEventRecord(ev[0], s));
      k_deriv<R, F><<<nb_site, kSiteThreads, 0, s>>>(c);
      CK(cudaEventRecord(ev[1], s));
      scalar(OP_THETA_MAIN, 2);
      CK(cudaEventRecord(ev[2], s));
      fft_xy(0, 0);
      CK(cudaEventRecord(ev[3], s));
      fft_zt();
      CK(cudaEventRecord(ev[4], s));
      fft_xy(1, 1);
      CK(cudaEventRecord(ev[5], s));
      scalar(OP_PR, 2);
      CK(cudaEventRecord(ev[6], s));
      probe<true>();
      CK(cudaEventRecord(ev[7], s));
      CK(cudaStreamSynchronize(s));
      float t[7];
      for (int k = 0; k < 7; k++) CK(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
      acc[0] += t[0];
      acc[6] += t[1] + t[5];
      acc[1] += t[2];
      acc[2] += t[3];
      acc[3] += t[4];
      acc[4] += t[6];
      CK(cudaEventRecord(ev[0], s));
      scalar(OP_PROBES, 2);
      CK(cudaEventRecord(ev[1], s));
      k_update<R, true, F><<<nb_site, kSiteThreads, 0, s>>>(c);
      CK(cudaEventRecord(ev[2], s));
      scalar(OP_END_CG, 0);
      CK(cudaEventRecord(ev[3], s));
      CK(cudaStreamSynchronize(s));
      for (int k = 0; k < 3; k++) CK(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
      acc[6] += t[0] + t[2];
      acc[5] += t[1];
      LAUNCHED(10);
    }
    for (auto &e : ev) cudaEventDestroy(e);
    // one complex number per site: of the links' type and of the fields'
    const double B = sizeof(cx<R>) * (double)V, BF = sizeof(cx<F>) * (double)V;
    // update: links in and out, the direction; with G (the FP32 phase of
    // mixed precision) also the accumulated transform in and out
    // (links: 4 kLinkCx complex numbers per site, their first two columns)
    const double L4 = 4.0 * kLinkCx;
    const double b[7] = {L4 * B + 4 * BF, 8 * BF, 8 * BF, 12 * BF,
                         L4 * B + 12 * BF,
                         (2 * L4 + (c.G ? 18 : 0)) * B + 4 * BF, 0.0};
    for (int k = 0; k < 7; k++) {
      ms[k] = acc[k] / n;
      if (bytes) bytes[k] = b[k];
    }
    return 0;
  }

  // ------------------------------------------------------------------
  // Coulomb: all slices as independent 3D problems (coulomb.cuh)
  CCtx<R> cc{};
  CoulState *d_cst = nullptr, *h_cst = nullptr;
  Slice *d_sl = nullptr, *h_sl = nullptr;
  double *d_ctraj = nullptr;
  int *d_cmask = nullptr;
  size_t ctraj_alloc = 0;
  int nbs = 0;
  cudaGraphExec_t gx_coul = nullptr;

  int cinit() {
    if (d_cst) return 0;
    const int T = c.L[3];
    nbs = (Lcu + kCoulThreads - 1) / kCoulThreads;
    CK(cudaMalloc(&d_cst, sizeof(CoulState)));
    CK(cudaMallocHost(&h_cst, sizeof(CoulState)));
    CK(cudaMalloc(&d_sl, sizeof(Slice) * T));
    CK(cudaMalloc(&d_cmask, sizeof(int) * T));
    c.skip = d_cmask;
    CK(cudaMallocHost(&h_sl, sizeof(Slice) * T));
    // per-slice partials: [T][nbs] pairs, next to the engine's own uses
    const size_t need = (size_t)T * nbs;
    const size_t have =
        std::max<size_t>((size_t)nb_site, (size_t)g_xy.x * g_xy.y) + 1024;
    if (need > have) {
      cudaFree(d_part);
      CK(cudaMalloc(&d_part, (need + 1024) * 2 * sizeof(double)));
      c.part = d_part;
    }
    cc.U = d_U;
    cc.g = d_G;
    cc.fb[0] = c.fb[0];
    cc.fb[1] = c.fb[1];
    cc.sb[0] = c.sb[0];
    cc.sb[1] = c.sb[1];
    cc.st = d_st;
    cc.cs = d_cst;
    cc.sl = d_sl;
    cc.part = d_part;
    for (int i = 0; i < 4; i++) cc.L[i] = c.L[i];
    cc.V = V;
    cc.Lcu = Lcu;
    cc.nbs = nbs;
    return 0;
  }

  void cscalar(int op) {
    const int T = c.L[3];
    k_cscalar<<<(T + kCScalarSlices - 1) / kCScalarSlices, 32 * kCScalarSlices, 0, s>>>(
        d_cst, d_sl, d_part, nbs, c.L[2], c.L[2] * T, op, (double)Lcu, d_st);
    LAUNCHED(1);
  }

  void capture_coul() {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
      cudaGetLastError();
      graph_ok = false;
      return;
    }
    const unsigned long long before = g_launches.load();
    citer();
    g_launches.store(before);
    if (cudaStreamEndCapture(s, &g) != cudaSuccess ||
        cudaGraphInstantiate(&gx_coul, g, 0) != cudaSuccess) {
      cudaGetLastError();
      gx_coul = nullptr;
      graph_ok = false;
    }
    if (g) cudaGraphDestroy(g);
  }

  // derivative and probes: FP64 storage one kernel each; FP32 storage an
  // FP32- and an FP64-arithmetic variant, each taking its own slices
  void cderiv(dim3 gs) {
    if (sizeof(R) == 8) {
      k_cderiv<R, double><<<gs, kCoulThreads, 0, s>>>(cc, SEL_ALWAYS);
    } else {
      k_cderiv<R, R><<<gs, kCoulThreads, 0, s>>>(cc, SEL_LOW);
      k_cderiv<R, double><<<gs, kCoulThreads, 0, s>>>(cc, SEL_HIGH);
      LAUNCHED(1);
    }
  }
  void cprobe(dim3 gs) {
    if (sizeof(R) == 8) {
      k_cprobe<R, double><<<gs, kCoulThreads, 0, s>>>(cc, SEL_ALWAYS);
    } else {
      k_cprobe<R, R><<<gs, kCoulThreads, 0, s>>>(cc, SEL_LOW);
      k_cprobe<R, double><<<gs, kCoulThreads, 0, s>>>(cc, SEL_HIGH);
      LAUNCHED(1);
    }
  }

  // one step of every live slice
  void citer() {
    const dim3 gs(nbs, c.L[3]);
    cderiv(gs);
    fft_xy(0, 0);
    fft_zt();
    fft_xy(1, 1);  // with the per-plane sums of the accelerated field
    cscalar(C_SUMS);
    cprobe(gs);
    cscalar(C_PROBES);
    k_cupdate<R><<<gs, kCoulThreads, 0, s>>>(cc);
    cscalar(C_END1);
    k_cmaint<R><<<gs, kCoulThreads, 0, s>>>(cc, 0);
    cscalar(C_END2);
    k_cmaint<R><<<gs, kCoulThreads, 0, s>>>(cc, 1);
    k_cflip<<<1, 1, 0, s>>>(d_st);
    LAUNCHED(6);
  }

  // GLU's Coulomb_FA (src/Gfix/CFACG.c:531-636) on the resident links
  // state of a new solve: every slice live, fields zero, g = 1 (or the g
  // left in place by an earlier phase)
  int cstart(const Params &p, bool identity = true) {
    if (cinit()) return -1;
    const int T = c.L[3];
    const size_t per = p.traj_cap ? p.traj_cap / T : 0;
    if (per && per * T > ctraj_alloc) {
      cudaFree(d_ctraj);
      CK(cudaMalloc(&d_ctraj, per * T * sizeof(double)));
      ctraj_alloc = per * T;
    }
    CoulState cst;
    memset(&cst, 0, sizeof cst);
    cst.gf_alpha = p.gf_alpha;
    cst.acc = p.acc;
    cst.cg_tol = 5E-11;
    cst.max_iters = (long long)p.max_iters;
    cst.facg = p.algo == GFIX_CG;
    cst.sd_fixed = p.sd_fixed;
    cst.active = T;
    cst.nslices = T;
    cst.seed = 0x5DEECE66Dull;
    cst.traj_cap = (int)per;
    cst.traj = per ? d_ctraj : nullptr;
    cst.done_mask = d_cmask;
    cst.prec_tol = sizeof(R) == 4 ? kPrecTolSingle : kPrecTol;
    // FP32 storage: FP32 arithmetic only while theta >= 1e-2 -- below it the
    // rounding of FP32 rotated links slows the slices' convergence (measured
    // on 32^3x64 and 64^3x128 slices), unlike the Landau probes (1e-5)
    cst.hp_below = 1E-2;
    cst.stall_window = p.stall_window;
    cst.stall_floor = p.stall_floor;
    cst.blowup = p.blowup;
    CK(cudaMemsetAsync(d_cmask, 0, sizeof(int) * T, s));
    CK(cudaMemcpyAsync(d_cst, &cst, sizeof cst, cudaMemcpyHostToDevice, s));
    std::vector<Slice> sl(T);
    memset(sl.data(), 0, sizeof(Slice) * T);
    for (auto &x : sl) {
      x.sd = 1;
      x.mode = SL_RUN;
      x.best_tr = 1e300;
    }
    CK(cudaMemcpyAsync(d_sl, sl.data(), sizeof(Slice) * T,
                       cudaMemcpyHostToDevice, s));
    DevState st;
    memset(&st, 0, sizeof st);
    CK(cudaMemcpyAsync(d_st, &st, sizeof st, cudaMemcpyHostToDevice, s));
    // in_old and sn start at zero (SD steps do not read them)
    CK(cudaMemsetAsync(c.fb[0], 0, (size_t)V * 16 * sizeof(cx<R>), s));
    if (identity) {
      k_cinit<R><<<(V + 255) / 256, 256, 0, s>>>(cc);
      LAUNCHED(1);
    }
    return 0;
  }

  // transform: 0 leaves the links untouched (a mixed-precision phase), 1
  // the slice transforms of a whole lattice, 2 all but the last slice's
  // temporal links (a block of slices of a larger lattice)
  int csolve(const Params &p, size_t *iters, double *slice_theta,
             size_t *slice_iters, size_t *traj_len, bool identity = true,
             int transform = 1) {
    if (cstart(p, identity)) return -1;
    const int T = c.L[3];
    const size_t per = p.traj_cap ? p.traj_cap / T : 0;
    // launches in citer() (FP32 storage: two variants of two kernels)
    const unsigned long long per_iter = sizeof(R) == 4 ? 15 : 13;
    int batch = 2;
    size_t guard = 0;
    const size_t limit = (p.max_iters + 2) * 9 * 64 + 1024;
    for (;;) {
      // the first steps run as direct launches (they load every kernel of
      // the sequence), the rest as replays of one captured step
      if (guard > 0 && !gx_coul && graph_ok) capture_coul();
      for (int k = 0; k < batch; k++) {
        if (gx_coul) {
          CK(cudaGraphLaunch(gx_coul, s));
          LAUNCHED(per_iter);
        } else {
          citer();
        }
      }
      CK(cudaGetLastError());
      if (read_state()) return -1;
      if (h_st->done) break;
      guard += batch;
      if (guard > limit)
        return fail("Coulomb solve did not stop after %zu steps", guard);
      batch = std::min(batch * 2, 32);
    }
    if (transform) {
      k_cslice_transform<R><<<(V + kCoulThreads - 1) / kCoulThreads,
                              kCoulThreads, 0, s>>>(cc, transform == 1);
      LAUNCHED(1);
    }
    CK(cudaMemcpyAsync(h_sl, d_sl, sizeof(Slice) * T, cudaMemcpyDeviceToHost,
                       s));
    CK(cudaStreamSynchronize(s));
    size_t tot = 0;
    for (int t = 0; t < T; t++) {
      tot += (size_t)h_sl[t].tot;
      if (slice_theta) slice_theta[t] = h_sl[t].tr;
      if (slice_iters) slice_iters[t] = (size_t)h_sl[t].tot;
    }
    *iters = tot;
    if (traj_len) *traj_len = 0;
    if (per && p.traj_theta) {
      // slice-major, stride per = traj_cap / Lt; unused entries are NaN
      std::vector<double> h(per * T);
      CK(cudaMemcpy(h.data(), d_ctraj, h.size() * sizeof(double),
                    cudaMemcpyDeviceToHost));
      for (int t = 0; t < T; t++)
        for (size_t k = 0; k < per; k++)
          p.traj_theta[t * per + k] =
              (int)k < h_sl[t].traj_len ? h[t * per + k] : NAN;
      if (traj_len) *traj_len = per * T;
    }
    return 0;
  }

  // Measurement aid: n steps of every slice (none may finish: accuracy 0)
  // with CUDA events between the launches; ms[k] = mean time of launch k:
  // 0 derivative, 1 xy FFT forward, 2 z FFT with psq, 3 xy FFT inverse +
  // sums, 4 direction + probes, 5 g update, 6 the scalar, housekeeping and
  // parity launches of a step; bytes[k] = its algorithmic HBM bytes.
  int profile_coul(const Params &p, int n, double *ms, double *bytes) {
    Params q = p;
    q.acc = 0.0;
    q.max_iters = (size_t)n + 16;
    q.traj_cap = 0;
    if (cstart(q)) return -1;
    const dim3 gs(nbs, c.L[3]);
    std::vector<cudaEvent_t> ev(10);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int it = 0; it < n; it++) {
      CK(cudaEventRecord(ev[0], s));
      cderiv(gs);
      CK(cudaEventRecord(ev[1], s));
      fft_xy(0, 0);
      CK(cudaEventRecord(ev[2], s));
      fft_zt();
      CK(cudaEventRecord(ev[3], s));
      fft_xy(1, 1);
      CK(cudaEventRecord(ev[4], s));
      cscalar(C_SUMS);
      CK(cudaEventRecord(ev[5], s));
      cprobe(gs);
      CK(cudaEventRecord(ev[6], s));
      cscalar(C_PROBES);
      CK(cudaEventRecord(ev[7], s));
      k_cupdate<R><<<gs, kCoulThreads, 0, s>>>(cc);
      CK(cudaEventRecord(ev[8], s));
      cscalar(C_END1);
      k_cmaint<R><<<gs, kCoulThreads, 0, s>>>(cc, 0);
      cscalar(C_END2);
      k_cmaint<R><<<gs, kCoulThreads, 0, s>>>(cc, 1);
      k_cflip<<<1, 1, 0, s>>>(d_st);
      CK(cudaEventRecord(ev[9], s));
      LAUNCHED(6);
      CK(cudaStreamSynchronize(s));
      float t[9];
      for (int k = 0; k < 9; k++) CK(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
      acc[0] += t[0];
      acc[1] += t[1];
      acc[2] += t[2];
      acc[3] += t[3];
      acc[4] += t[5];
      acc[5] += t[7];
      acc[6] += t[4] + t[6] + t[8];
    }
    for (auto &e : ev) cudaEventDestroy(e);
    CK(cudaGetLastError());
    const double B = sizeof(cx<R>) * (double)V;  // one complex per site
    // derivative: 3 links, g, 4 fields out; FFT passes: 4 fields in and out
    // (+ in_old for the sums); probes: in, sn_old, sn out, 3 links, g;
    // update: sn, g in and out
    const double L3 = 3.0 * kLinkCx;  // the three spatial links
    const double b[7] = {(L3 + 9 + 4) * B, 8 * B, 8 * B, 12 * B,
                         (4 + 4 + 4 + L3 + 9) * B, (4 + 9 + 9) * B, 0.0};
    for (int k = 0; k < 7; k++) {
      ms[k] = acc[k] / n;
      if (bytes) bytes[k] = b[k];
    }
    return 0;
  }

  // links: device AoS FP64 -> SoA R (and back)
  int from_aos(const double *aos) {
    k_aos_to_soa<R><<<(V + kTrSites - 1) / kTrSites, 256, 0, s>>>(aos, d_U, V);
    LAUNCHED(1);
    CK(cudaGetLastError());
    return 0;
  }
  int to_aos(double *aos) {
    k_soa_to_aos<R><<<(V + kTrSites - 1) / kTrSites, 256, 0, s>>>(d_U, aos, V);
    LAUNCHED(1);
    CK(cudaGetLastError());
    return 0;
  }
};

// ---------------------------------------------------------------------
// workspace cache: one engine per (device, shape, precision)

struct Key {
  int dev;
  size_t d[4];
  int prec;
  bool operator<(const Key &o) const {
    return std::tie(dev, d[0], d[1], d[2], d[3], prec) <
           std::tie(o.dev, o.d[0], o.d[1], o.d[2], o.d[3], o.prec);
  }
};

static std::map<Key, std::unique_ptr<Engine<double>>> g_e64;
static std::map<Key, std::unique_ptr<Engine<float>>> g_e32;

static Engine<double> *engine64(const size_t *d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail("no CUDA device");
    return nullptr;
  }
  Key k{dev, {d[0], d[1], d[2], d[3]}, 64};
  auto it = g_e64.find(k);
  if (it != g_e64.end()) return it->second.get();
  auto e = std::make_unique<Engine<double>>();
  if (e->init(d, false, true)) return nullptr;
  Engine<double> *p = e.get();
  g_e64[k] = std::move(e);
  return p;
}

// the FP64-link engine of mixed-precision solves: FP64 links, theta and
// updates, FP32 fields and FFT
static std::map<Key, std::unique_ptr<Engine<double, float>>> g_e64m;

static Engine<double, float> *engine64m(const size_t *d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail("no CUDA device");
    return nullptr;
  }
  Key k{dev, {d[0], d[1], d[2], d[3]}, 6432};
  auto it = g_e64m.find(k);
  if (it != g_e64m.end()) return it->second.get();
  auto e = std::make_unique<Engine<double, float>>();
  if (e->init(d, false, true)) return nullptr;
  Engine<double, float> *p = e.get();
  g_e64m[k] = std::move(e);
  return p;
}

static Engine<float> *engine32(const size_t *d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail("no CUDA device");
    return nullptr;
  }
  Key k{dev, {d[0], d[1], d[2], d[3]}, 32};
  auto it = g_e32.find(k);
  if (it != g_e32.end()) return it->second.get();
  auto e = std::make_unique<Engine<float>>();
  if (e->init(d, true, false)) return nullptr;
  Engine<float> *p = e.get();
  g_e32[k] = std::move(e);
  return p;
}

// Coulomb engines: FP64, with the slice gauge fields in d_G
static std::map<Key, std::unique_ptr<Engine<double>>> g_ec;

static Engine<double> *engine_coul(const size_t *d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail("no CUDA device");
    return nullptr;
  }
  Key k{dev, {d[0], d[1], d[2], d[3]}, 64};
  auto it = g_ec.find(k);
  if (it != g_ec.end()) return it->second.get();
  auto e = std::make_unique<Engine<double>>();
  if (e->init(d, true, true, true)) return nullptr;
  Engine<double> *p = e.get();
  g_ec[k] = std::move(e);
  return p;
}

static std::map<Key, std::unique_ptr<Engine<float>>> g_ec32;

static Engine<float> *engine_coul32(const size_t *d) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail("no CUDA device");
    return nullptr;
  }
  Key k{dev, {d[0], d[1], d[2], d[3]}, 32};
  auto it = g_ec32.find(k);
  if (it != g_ec32.end()) return it->second.get();
  auto e = std::make_unique<Engine<float>>();
  if (e->init(d, true, false, true)) return nullptr;
  Engine<float> *p = e.get();
  g_ec32[k] = std::move(e);
  return p;
}

static Params to_params(const gfix_params *p) {
  Params q;
  q.gf_alpha = p->gf_alpha;
  q.acc = p->accuracy;
  q.max_iters = p->max_iters;
  q.algo = p->algo;
  q.sd_fixed = p->sd_fixed_step;
  q.traj_theta = p->traj_theta;
  q.traj_func = p->traj_func;
  q.traj_cap = p->traj_cap;
  return q;
}

// Landau solve of the links staged (AoS FP64) in e64->d_aos
// Mixed precision hand-over from the FP32 phase (engine f, finished, it32
// iterations, theta th32) to the FP64 engine e: U64 <- G U64 G^dag with the
// accumulated G reunitarised in FP64; for FACG the FP32 run's last direction
// and accelerated derivative become the FP64 run's sn_old / in_old, so the
// conjugate directions continue across the switch.  A phase that ended
// non-finite hands over nothing (FP64 from the staged input links; it32 = 0,
// *restart = 1).
// The links a Landau attempt starts from: the staged input (AoS FP64 in
// d_aos); for a restart (attempt > 0) randomly gauge transformed, as GLU's
// Landau driver re-reads its input and applies random_transform
// (src/Gfix/Landau.c:241-257, src/Geometry/random_config.c:107-120).
template <typename E>
static int stage_input(E *e, unsigned long long seed, int attempt) {
  if (e->from_aos(e->d_aos)) return -1;
  if (attempt > 0) {
    k_random_transform<<<e->nb_site, kSiteThreads, 0, e->s>>>(e->c, seed, attempt);
    LAUNCHED(1);
    CK(cudaGetLastError());
  }
  return 0;
}

// E: the FP64-link engine of the second phase (FP64 or FP32 fields)
template <typename E>
static int mixed_handover(E *e, Engine<float> *f, const Params &p64,
                          size_t *it32, double th32, int *restart,
                          unsigned long long seed, int attempt) {
  *restart = 0;
  if (!(*it32 == kSentinel || *it32 > 0)) return 0;
  // the FP32 phase's G, widened and reunitarised in FP64, on the FP64 links
  CK(cudaStreamSynchronize(f->s));
  k_apply_gauge<<<e->nb_site, kSiteThreads, 0, e->s>>>(e->c, (const cx<float> *)f->d_G);
  LAUNCHED(1);
  double tt = 0.0;
  if (e->reset(p64) || e->theta_test(&tt)) return -1;
  if (!std::isfinite(th32) || !std::isfinite(tt)) {
    if (stage_input(e, seed, attempt)) return -1;
    *it32 = 0;
    *restart = 1;
    return 0;
  }
  if (p64.algo == GFIX_CG && *it32 != kSentinel) {
    // f's state after its last iteration: in_old = fb[parity ^ 1] (the END
    // step flipped it), sn_old = sb[sparity]
    if (f->read_state()) return -1;
    const cx<float> *in_old = f->c.fb[f->h_st->parity ^ 1];
    const cx<float> *sn_old = f->c.sb[f->h_st->sparity];
    k_convert<<<1184, 256, 0, e->s>>>(in_old, e->c.fb[1], (size_t)e->V * 4);
    k_convert<<<1184, 256, 0, e->s>>>(sn_old, e->c.sb[0], (size_t)e->V * 4);
    LAUNCHED(2);
    CK(cudaStreamSynchronize(e->s));
    e->warm = true;
    e->warm_inold = f->h_st->inold;
  }
  return 0;
}

// One Landau solve (GLU's FACG / FASD, or the mixed-precision pair of
// them) of the links resident in e64's SoA buffer, to the accuracy and
// iteration bound of p; the fixed links are left there.  attempt: the
// random restart whose start a failed mixed first phase goes back to.
template <typename E>
static int solve_resident(E *e64, const gfix_params *gp, const Params &p,
                          int attempt, gfix_result *r) {
  gfix_result res;
  memset(&res, 0, sizeof res);
  size_t iters = 0;
  double th = 0.0;
  size_t tl = 0;
  if (gp->precision == GFIX_MIXED) {
    // FP32 phase on a converted copy, tracking the gauge transform G
    Engine<float> *e32 = engine32(e64->dims);
    if (!e32) return -1;
    // e32 runs on e64's stream order: synchronise the two streams
    CK(cudaStreamSynchronize(e64->s));
    const size_t n = (size_t)e64->V * 4 * kLinkCx;
    k_convert<double, float><<<1184, 256, 0, e32->s>>>(e64->d_U, e32->d_U, n);
    k_identity<float><<<(e64->V + 255) / 256, 256, 0, e32->s>>>(e32->d_G,
                                                                e64->V);
    LAUNCHED(2);
    Params p32 = p;
    p32.acc = std::max(gp->switch_theta, gp->accuracy);
    stall_rule(p32);
    size_t it32 = 0;
    double th32 = 0.0;
    if (e32->solve(p32, &it32, &th32)) return -1;
    size_t tl32 = 0;
    if (e32->fetch_traj(p32, &tl32)) return -1;
    {
      int restart = 0;
      if (mixed_handover(e64, e32, p, &it32, th32, &restart, gp->restart_seed,
                         attempt))
        return -1;
      if (restart) {
        tl32 = 0;
        res.restarts++;
      }
    }
    res.iters_fp32 = (it32 == kSentinel) ? p32.max_iters : it32;
    Params p64 = p;
    if (p.traj_cap) {
      p64.traj_theta = p.traj_theta ? p.traj_theta + tl32 : nullptr;
      p64.traj_func = p.traj_func ? p.traj_func + tl32 : nullptr;
      p64.traj_cap = p.traj_cap > tl32 ? p.traj_cap - tl32 : 0;
    }
    size_t it64 = 0;
    if (e64->solve(p64, &it64, &th)) return -1;
    if (e64->fetch_traj(p64, &tl)) return -1;
    tl += tl32;
    iters = (it64 == kSentinel) ? kSentinel : res.iters_fp32 + it64;
  } else {
    if (e64->solve(p, &iters, &th)) return -1;
    if (e64->fetch_traj(p, &tl)) return -1;
  }
  res.iters = iters;
  res.theta = th;
  res.traj_len = tl;
  *r = res;
  return 0;
}

// GLU's Landau driver prints every failed attempt (print_failure_info,
// src/Gfix/Landau.c:70-86) and every gauge copy; the flat entry points
// stay silent
static thread_local bool t_restart_log = false;
void set_restart_log(bool on) { t_restart_log = on; }

// GLU's luxury_copy_fast (src/Gfix/Landau.c:92-211, compiled in with
// LUXURY_GAUGE): gp->luxury_copies random gauge copies of the attempt's
// start, each fixed to theta < 1e-6 in at most 1000 iterations; of the
// copies that converged within the bound, the one with the largest gauge
// functional is kept -- the smallest with gp->luxury_best (GLU's
// BEST_COPY) -- and fixed to the requested accuracy.  The count is GLU's:
// the last copy's iterations plus the final fix's.  Copies are transformed
// by this library's generator; if no copy is kept, the final fix starts
// from the attempt's start (GLU's would start from an unset lattice).
template <typename E>
static int luxury_resident(E *e64, const gfix_params *gp, int attempt,
                           gfix_result *r) {
  constexpr double kCopyAcc = 1E-6;    // Landau.c:142
  constexpr size_t kCopyMax = 1000;    // Landau.c:143
  Params pc = to_params(gp);
  pc.acc = kCopyAcc;
  pc.max_iters = kCopyMax;
  pc.traj_cap = 0;
  pc.traj_theta = pc.traj_func = nullptr;
  gfix_params gc = *gp;
  gc.accuracy = kCopyAcc;
  gc.max_iters = kCopyMax;
  gc.traj_cap = 0;
  gc.traj_theta = gc.traj_func = nullptr;
  if (!e64->d_best)
    CK(cudaMalloc(&e64->d_best, (size_t)e64->V * 4 * kLinkCx * sizeof(cx<double>)));
  const size_t bytes = (size_t)e64->V * 4 * kLinkCx * sizeof(cx<double>);
  double keep = gp->luxury_best ? 1.0 : 0.0;  // Landau.c:122-126
  bool kept = false;
  size_t iters = 0;
  int restarts = 0;
  for (int copy = 0; copy < gp->luxury_copies; copy++) {
    if (stage_input(e64, gp->restart_seed, attempt)) return -1;
    const int id = (1 << 20) + attempt * 4096 + copy;  // distinct from restarts
    k_random_transform<<<e64->nb_site, kSiteThreads, 0, e64->s>>>(
        e64->c, gp->restart_seed, id);
    LAUNCHED(1);
    gfix_result rc;
    if (solve_resident(e64, &gc, pc, attempt, &rc)) return -1;
    restarts += rc.restarts;
    iters = rc.iters;
    double tt = 0.0;
    Params q;
    if (e64->reset(q) || e64->theta_test(&tt)) return -1;
    const double f = e64->h_st->func;  // gauge_functional of the copy
    const bool ok = iters != kCopyMax && iters != kSentinel &&
                    (gp->luxury_best ? f < keep : f > keep);
    if (t_restart_log)
      fprintf(stdout, "  [COPY] %d [FUNCTIONAL] %1.15f [ITER] %zu %s", copy, f,
              iters, ok ? " -> Copy accepted\n" : "");
    if (ok) {
      keep = f;
      kept = true;
      CK(cudaMemcpyAsync(e64->d_best, e64->d_U, bytes, cudaMemcpyDeviceToDevice,
                         e64->s));
    } else if (t_restart_log) {
      fprintf(stdout, " -> Copy rejected %e\n", f - keep);
    }
  }
  if (kept) {
    CK(cudaMemcpyAsync(e64->d_U, e64->d_best, bytes, cudaMemcpyDeviceToDevice, e64->s));
  } else if (stage_input(e64, gp->restart_seed, attempt)) {
    return -1;
  }
  gfix_result rf;
  if (solve_resident(e64, gp, to_params(gp), attempt, &rf)) return -1;
  rf.iters = rf.iters + iters;  // Landau.c:187-191: added to the last copy's
  rf.restarts += restarts;
  *r = rf;
  return 0;
}

// One Landau attempt: the staged input (a restart's random transform of it
// for attempt > 0), then GLU's solve or its luxury copies
template <typename E>
static int landau_attempt(E *e64, const gfix_params *gp, int attempt,
                          gfix_result *r) {
  if (stage_input(e64, gp->restart_seed, attempt)) return -1;
  if (gp->luxury_copies > 0) return luxury_resident(e64, gp, attempt, r);
  return solve_resident(e64, gp, to_params(gp), attempt, r);
}

// A Landau fix of the links staged in e64->d_aos, with GLU's random
// restarts (src/Gfix/Landau.c:303-340) when p->max_restarts > 0: after a
// failed solve (the sentinel) the input is randomly gauge transformed and
// solved again, up to max_restarts times.  The count follows GLU's sums:
// the first attempt's sentinel, + max_iters per failed restart, + the
// successful attempt's count; GLU_FAILURE when every attempt failed.  The
// fixed links are left in e64's SoA links (resident) and in d_aos.
template <typename E>
static int landau_staged(E *e64, const gfix_params *gp, gfix_result *r) {
  CK(cudaEventRecord(e64->ev0, e64->s));
  gfix_result res;
  if (landau_attempt(e64, gp, 0, &res)) return -1;
  if (res.iters == kSentinel && gp->max_restarts > 0) {
    if (t_restart_log)
      fprintf(stderr, "\n[GF] Non-convergence ... Randomly-restarting \n"
              "\n[GF] Failure :: %d || Iters :: %zu || ACC :: %e \n", 0,
              gp->max_iters, res.theta);
    size_t total = kSentinel;
    int failure = 1;
    for (; failure <= gp->max_restarts; failure++) {
      gfix_result a;
      if (landau_attempt(e64, gp, failure, &a)) return -1;
      a.restarts += res.restarts + 1;
      res = a;
      if (a.iters != kSentinel) {
        total += a.iters;
        break;
      }
      total += gp->max_iters;
      if (t_restart_log)
        fprintf(stderr, "\n[GF] Non-convergence ... Randomly-restarting \n"
                "\n[GF] Failure :: %d || Iters :: %zu || ACC :: %e \n",
                failure, a.iters, a.theta);
    }
    res.iters = failure > gp->max_restarts ? kGluFailure : total;
  }
  CK(cudaEventRecord(e64->ev1, e64->s));
  if (e64->to_aos(e64->d_aos)) return -1;
  CK(cudaStreamSynchronize(e64->s));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e64->ev0, e64->ev1));
  res.gpu_ms = ms;
  if (r) *r = res;
  return 0;
}

// n configurations of one shape fixed one after another by one engine
// (each as landau_staged, results r[0..n-1]), the host links of the next
// configuration crossing to the device, and those of the previous one back,
// on a copy stream while the current one is being solved.  The engine's AoS
// buffer alternates with a second one: configuration i is staged into
// buffer i % 2, whose previous contents (configuration i - 2) left it
// earlier on the same copy stream.
template <typename E>
static int sequence_staged(E *e, double *const *links, size_t n,
                           const gfix_params *gp, gfix_result *r) {
  const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
  if (!e->d_aos2) CK(cudaMalloc(&e->d_aos2, bytes));
  if (!e->s_copy) {
    CK(cudaStreamCreateWithFlags(&e->s_copy, cudaStreamNonBlocking));
    for (cudaEvent_t &ev : e->ev_in)
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&e->ev_solved, cudaEventDisableTiming));
  }
  double *const buf[2] = {e->d_aos, e->d_aos2};
  CK(cudaStreamSynchronize(e->s));
  CK(cudaMemcpyAsync(buf[0], links[0], bytes, cudaMemcpyHostToDevice, e->s_copy));
  CK(cudaEventRecord(e->ev_in[0], e->s_copy));
  int rc = 0;
  for (size_t i = 0; i < n && rc == 0; i++) {
    const int j = (int)(i & 1);
    if (i + 1 < n) {
      CK(cudaMemcpyAsync(buf[j ^ 1], links[i + 1], bytes, cudaMemcpyHostToDevice,
                         e->s_copy));
      CK(cudaEventRecord(e->ev_in[j ^ 1], e->s_copy));
    }
    CK(cudaStreamWaitEvent(e->s, e->ev_in[j], 0));
    e->d_aos = buf[j];
    rc = landau_staged(e, gp, &r[i]);
    e->d_aos = buf[0];
    if (rc) break;
    CK(cudaEventRecord(e->ev_solved, e->s));
    CK(cudaStreamWaitEvent(e->s_copy, e->ev_solved, 0));
    CK(cudaMemcpyAsync(links[i], buf[j], bytes, cudaMemcpyDeviceToHost, e->s_copy));
  }
  CK(cudaStreamSynchronize(e->s_copy));
  return rc;
}

// ---------------------------------------------------------------------
// Batches: many configurations, of any shapes, fixed together.  Every
// configuration keeps its own engine (buffers, device control block,
// iteration graph); one parent CUDA graph holds the iteration graph of every
// unfinished configuration as a child, so one launch advances all of them
// at once, concurrently.  A configuration that has converged turns its
// kernels into no-ops through its own done flag (the per-instance mask);
// the parent graph is rebuilt without it once a quarter of the live set has
// finished.  Each configuration runs exactly the kernel sequence of a solve
// of its own, so its results are those of gfix_landau.

template <typename E>
static int batch_solve(std::vector<E *> &es, const Params &p,
                       std::vector<size_t> &iters, std::vector<double> &th,
                       cudaStream_t bs) {
  const size_t n = es.size();
  std::vector<char> fin(n, 0);
  iters.assign(n, 0);
  th.assign(n, 0.0);
  bool graphs = true;
  for (size_t i = 0; i < n; i++) {
    bool f = false;
    if (es[i]->run_start(p, &f, &iters[i], &th[i])) return -1;
    fin[i] = f;
    graphs &= es[i]->run_exec() != nullptr && es[i]->run_graph() != nullptr;
  }
  if (!graphs) {
    // no graphs: one configuration after the other
    for (size_t i = 0; i < n; i++) {
      bool f = fin[i] != 0;
      while (!f) {
        if (es[i]->replay(es[i]->run_exec(), es[i]->run_cg, p.sd_fixed != 0))
          return -1;
        if (es[i]->run_after(&f, &iters[i], &th[i])) return -1;
      }
    }
    return 0;
  }
  std::vector<cudaEvent_t> ev(n, nullptr);
  for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaGraphExec_t px = nullptr;
  size_t built_live = 0, guard = 0;
  unsigned long long per_replay = 0;
  int batch = 2;
  int rc = 0;
  for (;;) {
    std::vector<size_t> live;
    for (size_t i = 0; i < n; i++)
      if (!fin[i]) live.push_back(i);
    if (live.empty()) break;
    if (!px || live.size() * 4 <= built_live * 3) {
      if (px) cudaGraphExecDestroy(px);
      px = nullptr;
      cudaGraph_t pg = nullptr;
      per_replay = 0;
      if (cudaGraphCreate(&pg, 0) != cudaSuccess) { rc = fail("graph create"); break; }
      for (size_t i : live) {
        cudaGraphNode_t node;
        if (cudaGraphAddChildGraphNode(&node, pg, nullptr, 0,
                                       es[i]->run_graph()) != cudaSuccess) {
          rc = fail("child graph node: %s", cudaGetErrorString(cudaGetLastError()));
          break;
        }
        per_replay += es[i]->per_iter_launches(es[i]->run_cg, p.sd_fixed != 0);
      }
      if (!rc && cudaGraphInstantiate(&px, pg, 0) != cudaSuccess) {
        rc = fail("batch graph instantiate: %s",
                  cudaGetErrorString(cudaGetLastError()));
      }
      cudaGraphDestroy(pg);
      if (rc) break;
      built_live = live.size();
    }
    // the heads of new runs were launched on the engines' own streams
    for (size_t i : live) {
      CK(cudaEventRecord(ev[i], es[i]->s));
      CK(cudaStreamWaitEvent(bs, ev[i], 0));
    }
    for (int k = 0; k < batch; k++) {
      CK(cudaGraphLaunch(px, bs));
      LAUNCHED(per_replay);
    }
    for (size_t i : live)
      CK(cudaMemcpyAsync(es[i]->h_st, es[i]->d_st, sizeof(DevState),
                         cudaMemcpyDeviceToHost, bs));
    CK(cudaStreamSynchronize(bs));
    for (size_t i : live) {
      if (!es[i]->h_st->done) continue;
      bool f = false;
      if (es[i]->run_after(&f, &iters[i], &th[i])) { rc = -1; break; }
      fin[i] = f;
    }
    if (rc) break;
    guard += batch;
    if (guard > (size_t)p.max_iters * 64 + 1024) {
      rc = fail("batch did not stop after %zu iterations", guard);
      break;
    }
    batch = std::min(batch * 2, 32);
  }
  if (px) cudaGraphExecDestroy(px);
  for (auto &e : ev) cudaEventDestroy(e);
  return rc;
}

struct BatchInst {
  size_t dims[4];
  double *links = nullptr;  // host or device, double[V][4][9][2]
  bool device = false;
  std::unique_ptr<Engine<double>> e64;           // GFIX_FP64
  std::unique_ptr<Engine<double, float>> e64m;   // GFIX_MIXED: FP64 links
  std::unique_ptr<Engine<float>> e32;            //   and the FP32 phase
  gfix_result res;
  Engine<double> *fp64(Engine<double> *) { return e64.get(); }
  Engine<double, float> *fp64(Engine<double, float> *) { return e64m.get(); }
};

struct Batch {
  gfix_params p;
  std::vector<std::unique_ptr<BatchInst>> inst;
  cudaStream_t bs = nullptr;
  ~Batch() {
    inst.clear();
    if (bs) cudaStreamDestroy(bs);
  }
};

// mixed precision for a whole batch, phase by phase as landau_staged does
// it for one configuration
// E: the FP64-link engine type of the batch's precision
template <typename E>
static int batch_run_t(Batch *b) {
  const Params p = to_params(&b->p);
  const size_t n = b->inst.size();
  if (!n) return 0;
  if (!b->bs) CK(cudaStreamCreateWithFlags(&b->bs, cudaStreamNonBlocking));
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  CK(cudaDeviceSynchronize());
  CK(cudaEventRecord(t0, b->bs));
  std::vector<E *> e64(n);
  for (size_t i = 0; i < n; i++) {
    BatchInst &I = *b->inst[i];
    memset(&I.res, 0, sizeof I.res);
    E *e = I.fp64((E *)nullptr);
    e64[i] = e;
    const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
    CK(cudaMemcpyAsync(e->d_aos, I.links, bytes,
                       I.device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       e->s));
    if (e->from_aos(e->d_aos)) return -1;
  }
  std::vector<size_t> it32(n, 0), it64;
  std::vector<double> th32(n, 0.0), th64;
  Params p64 = p;
  p64.traj_cap = 0;
  if (b->p.precision == GFIX_MIXED) {
    std::vector<Engine<float> *> e32(n);
    for (size_t i = 0; i < n; i++) {
      BatchInst &I = *b->inst[i];
      if (!I.e32) {
        I.e32 = std::make_unique<Engine<float>>();
        if (I.e32->init(I.dims, true, false)) return -1;
      }
      e32[i] = I.e32.get();
      CK(cudaStreamSynchronize(e64[i]->s));
      k_convert<double, float><<<1184, 256, 0, e32[i]->s>>>(
          e64[i]->d_U, e32[i]->d_U, (size_t)e64[i]->V * 4 * kLinkCx);
      k_identity<float><<<(e64[i]->V + 255) / 256, 256, 0, e32[i]->s>>>(
          e32[i]->d_G, e64[i]->V);
      LAUNCHED(2);
    }
    Params p32 = p64;
    p32.acc = std::max(b->p.switch_theta, b->p.accuracy);
    stall_rule(p32);
    if (batch_solve(e32, p32, it32, th32, b->bs)) return -1;
    for (size_t i = 0; i < n; i++) {
      int restart = 0;
      // (batches make no random restarts: attempt 0 only)
      if (mixed_handover(e64[i], e32[i], p64, &it32[i], th32[i], &restart, 0, 0))
        return -1;
      b->inst[i]->res.restarts += restart;
    }
  }
  if (batch_solve(e64, p64, it64, th64, b->bs)) return -1;
  for (size_t i = 0; i < n; i++) {
    BatchInst &I = *b->inst[i];
    E *e = e64[i];
    if (e->to_aos(e->d_aos)) return -1;
    const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
    CK(cudaMemcpyAsync(I.links, e->d_aos, bytes,
                       I.device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       e->s));
    const size_t f32 = (it32[i] == kSentinel) ? p.max_iters : it32[i];
    I.res.iters_fp32 = b->p.precision == GFIX_MIXED ? f32 : 0;
    I.res.iters = it64[i] == kSentinel ? kSentinel : I.res.iters_fp32 + it64[i];
    I.res.theta = th64[i];
  }
  for (size_t i = 0; i < n; i++) {
    CK(cudaEventRecord(e64[i]->ev1, e64[i]->s));
    CK(cudaStreamWaitEvent(b->bs, e64[i]->ev1, 0));
  }
  CK(cudaEventRecord(t1, b->bs));
  CK(cudaEventSynchronize(t1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, t0, t1));
  for (auto &I : b->inst) I->res.gpu_ms = ms;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  return 0;
}

static int batch_run(Batch *b) {
  return b->p.precision == GFIX_MIXED ? batch_run_t<Engine<double, float>>(b)
                                      : batch_run_t<Engine<double>>(b);
}

}  // namespace gfix

using namespace gfix;

// ---------------------------------------------------------------------
// flat C ABI

extern "C" {

const char *gfix_last_error(void) { return g_err.c_str(); }

unsigned long long gfix_kernel_launches(void) { return g_launches.load(); }

void gfix_fft_tuning(int on) {
  g_fft_tune = on ? 1 : 0;
  // workspaces built under the other setting are rebuilt at next use
  g_e64.clear();
  g_e32.clear();
  g_ec.clear();
  g_ec32.clear();
}

int gfix_fft_plan(const size_t dims[4], int coulomb, int precision, int *plan,
                  float *ms) {
  if (!dims || !plan) return fail("null argument");
  for (int i = 0; i < 4; i++)
    if (dims[i] < 2) return fail("extent %zu of dimension %d below 2", dims[i], i);
  auto get = [&](auto *e) {
    plan[0] = e->xy_plan;
    plan[1] = e->c.zt_b;
    plan[2] = e->zt_plan;
    if (ms) {
      ms[0] = ms[1] = 0.f;
      const auto key = std::make_tuple(e->c.L[0], e->c.L[1], e->c.L[2],
                                       e->c.L[3], e->coul);
      auto it = e->tuned().find(key);
      if (it != e->tuned().end()) {
        ms[0] = it->second.xy_ms;
        ms[1] = it->second.zt_ms;
      }
    }
    return 0;
  };
  if (precision == GFIX_MIXED) {
    if (coulomb) {
      Engine<float> *f = engine_coul32(dims);
      return f ? get(f) : -1;
    }
    Engine<float> *f = engine32(dims);
    return f ? get(f) : -1;
  }
  Engine<double> *e = coulomb ? engine_coul(dims) : engine64(dims);
  return e ? get(e) : -1;
}

void gfix_release(void) {
  gfix_cuts_release();
  gfix_update_release();
  g_e64.clear();
  g_e64m.clear();
  g_e32.clear();
  g_ec.clear();
  g_ec32.clear();
}

static int check_params(const size_t *dims, const gfix_params *p) {
  if (!dims || !p) return fail("null dims or params");
  for (int i = 0; i < 4; i++)
    if (dims[i] < 2) return fail("extent %zu of dimension %d below 2", dims[i], i);
  if (p->algo != GFIX_CG && p->algo != GFIX_SD) return fail("unknown algo %d", p->algo);
  if (p->precision != GFIX_FP64 && p->precision != GFIX_MIXED)
    return fail("unknown precision %d", p->precision);
  if (p->traj_cap && !p->traj_theta) return fail("traj_cap without traj_theta");
  if (p->max_restarts < 0) return fail("max_restarts %d below 0", p->max_restarts);
  if (p->luxury_copies < 0) return fail("luxury_copies %d below 0", p->luxury_copies);
  return 0;
}

}  // extern "C"

namespace gfix {

int cuda_failure(const char *what, cudaError_t e) {
  return fail("%s: %s", what, cudaGetErrorString(e));
}

static thread_local PhaseMark t_mark = nullptr;
static thread_local void *t_mark_ctx = nullptr;
void set_phase_mark(PhaseMark fn, void *ctx) {
  t_mark = fn;
  t_mark_ctx = ctx;
}
// the phase's work complete on s, then the caller's mark
static int mark(cudaStream_t s, const char *phase) {
  if (!t_mark) return 0;
  CK(cudaStreamSynchronize(s));
  t_mark(t_mark_ctx, phase);
  return 0;
}

}  // namespace gfix

namespace {
// the links of the flat entry points: one contiguous host array
struct HostArray final : gfix::LinkIO {
  double *links;
  explicit HostArray(double *l) : links(l) {}
  int to_device(double *d_aos, size_t V, cudaStream_t s) override {
    CK(cudaMemcpyAsync(d_aos, links, V * 36 * sizeof(double2),
                       cudaMemcpyHostToDevice, s));
    return 0;
  }
  int to_host(const double *d_aos, size_t V, cudaStream_t s) override {
    CK(cudaMemcpyAsync(links, d_aos, V * 36 * sizeof(double2),
                       cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return 0;
  }
};
}  // namespace

// The engine that stages a Landau solve's links and runs its FP64-link
// phase: FP64 fields under GFIX_FP64, FP32 fields under GFIX_MIXED (whose
// FP32 phase runs on a further, all-FP32 engine)
template <typename Fn>
static int with_landau_engine(const size_t *dims, int precision, Fn &&fn) {
  if (precision == GFIX_MIXED) {
    Engine<double, float> *e = engine64m(dims);
    return e ? fn(e) : -1;
  }
  Engine<double> *e = engine64(dims);
  return e ? fn(e) : -1;
}

extern "C" {

int gfix_landau(double *links, const size_t dims[4], const gfix_params *p,
                gfix_result *r) {
  if (check_params(dims, p)) return -1;
  if (!links) return fail("null links");
  HostArray io(links);
  return gfix::landau_io(io, dims, p, r);
}

int gfix_landau_sequence(double *const *links, size_t n, const size_t dims[4],
                         const gfix_params *p, gfix_result *r) {
  if (check_params(dims, p)) return -1;
  if (n == 0) return 0;
  if (!links || !r) return fail("null argument");
  for (size_t i = 0; i < n; i++)
    if (!links[i]) return fail("null links of configuration %zu", i);
  return with_landau_engine(dims, p->precision, [&](auto *e) -> int {
    if (p->precision == GFIX_MIXED && !engine32(dims)) return -1;
    return sequence_staged(e, links, n, p, r);
  });
}

int gfix_landau_device(double *d_links, const size_t dims[4],
                       const gfix_params *p, gfix_result *r) {
  if (check_params(dims, p)) return -1;
  if (!d_links) return fail("null links");
  return with_landau_engine(dims, p->precision, [&](auto *e) -> int {
    const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
    // the caller's buffer is on the legacy default stream order
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpyAsync(e->d_aos, d_links, bytes, cudaMemcpyDeviceToDevice, e->s));
    if (landau_staged(e, p, r)) return -1;
    CK(cudaMemcpyAsync(d_links, e->d_aos, bytes, cudaMemcpyDeviceToDevice, e->s));
    CK(cudaStreamSynchronize(e->s));
    return 0;
  });
}

// (templates: C++ linkage inside the C ABI block)
extern "C++" {

// theta_test_lin, functional and plaquette of the links resident in e's
// SoA buffer (out[0..2])
template <typename E>
static int observables_resident(E *e, double *out) {
  Params p;
  if (e->reset(p)) return -1;
  double tt = 0;
  if (e->theta_test(&tt)) return -1;
  // theta_test leaves the functional sum of the same links in func
  out[0] = tt;
  out[1] = e->h_st->func;
  k_plaquette<<<e->nb_site, kSiteThreads, 0, e->s>>>(e->c);
  LAUNCHED(1);
  std::vector<double> part(e->nb_site);
  CK(cudaMemcpyAsync(part.data(), e->d_part, part.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, e->s));
  CK(cudaStreamSynchronize(e->s));
  double sum = 0.0;
  for (double v : part) sum += v;
  out[2] = 2.0 * sum / (3.0 * 4 * 3 * (double)e->V);
  return 0;
}

// host links -> e's AoS staging -> e's SoA links
template <typename E>
static int stage_host(E *e, const double *links) {
  const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
  CK(cudaMemcpyAsync(e->d_aos, links, bytes, cudaMemcpyHostToDevice, e->s));
  return e->from_aos(e->d_aos);
}

// GLU's post-fix link diagnostics of the links resident in e (out[0..5],
// as gfix_link_diagnostics)
template <typename E>
static int diagnostics_resident(E *e, double *out) {
  const int T = e->c.L[3], lcu = e->V / T;
  const int nbs = (lcu + kDiagThreads - 1) / kDiagThreads;
  std::vector<double> part((size_t)kDiagVals * nbs * T);
  double *d_p = nullptr;
  CK(cudaMalloc(&d_p, part.size() * sizeof(double)));
  auto c = e->c;
  c.part = d_p;
  k_link_diag<<<dim3(nbs, T), kDiagThreads, 0, e->s>>>(c, lcu, nbs);
  LAUNCHED(1);
  CK(cudaMemcpyAsync(part.data(), d_p, part.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, e->s));
  CK(cudaStreamSynchronize(e->s));
  cudaFree(d_p);
  // fixed-order sums; const_time: per slice t >= 1 the differences of the
  // Hermitian-projection sums from slice 0 (gftests.c:84-95)
  double sp = 0.0, tl = 0.0, mx = -1e300;
  std::vector<std::array<double, 16>> hs(T);  // linear 8 reals, log 8 reals
  for (int t = 0; t < T; t++) {
    hs[t].fill(0.0);
    for (int b = 0; b < nbs; b++) {
      const double *q = &part[(size_t)kDiagVals * ((size_t)t * nbs + b)];
      sp += q[0];
      tl += q[1];
      mx = std::max(mx, q[2]);
      for (int k = 0; k < 16; k++) hs[t][k] += q[3 + k];
    }
  }
  double av = 0.0, avlog = 0.0;
  for (int t = 1; t < T; t++) {
    for (int d = 0; d < 2; d++) {
      const double *a = hs[0].data() + 8 * d, *b = hs[t].data() + 8 * d;
      double x = std::fabs(a[0] - b[0]);
      x += std::hypot(a[1] - b[1], a[2] - b[2]);
      x += std::hypot(a[3] - b[3], a[4] - b[4]);
      x += std::fabs(a[5] - b[5]);
      x += std::hypot(a[6] - b[6], a[7] - b[7]);
      (d ? avlog : av) += x;
    }
  }
  const double V = (double)e->V;
  out[0] = sp / (3.0 * 3.0 * V);        // all_links: spatial
  out[1] = tl / (3.0 * V);              //            temporal
  out[2] = (sp + tl) / (4.0 * 3.0 * V); // indivlinks average
  out[3] = mx / 3.0;                    // largest Re tr / NC
  out[4] = T > 1 ? av / (9.0 * (T - 1)) : 0.0;     // const_time, linear
  out[5] = T > 1 ? avlog / (9.0 * (T - 1)) : 0.0;  //             logarithmic
  return 0;
}

// gf_check of the links resident in e: out[0..9] as gfix_gf_check
template <typename E>
static int gf_check_resident(E *e, double *out) {
  const int nb = e->nb_site;
  double *d_p = nullptr;
  CK(cudaMalloc(&d_p, (size_t)nb * kGfcVals * sizeof(double)));
  auto c = e->c;
  c.part = d_p;
  k_gf_check<<<nb, kSiteThreads, 0, e->s>>>(c);
  LAUNCHED(1);
  std::vector<double> part((size_t)nb * kGfcVals);
  const cudaError_t err = cudaMemcpyAsync(part.data(), d_p, part.size() * sizeof(double),
                                          cudaMemcpyDeviceToHost, e->s);
  const cudaError_t err2 = cudaStreamSynchronize(e->s);
  cudaFree(d_p);
  CK(err);
  CK(err2);
  // fixed-order sums; theta = 2 sum / (NC V) (gftests.c:249, :289)
  double sum[4] = {0, 0, 0, 0}, mx[4] = {0, 0, 0, 0};
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 4; k++) {
      sum[k] += part[(size_t)b * kGfcVals + k];
      mx[k] = std::max(mx[k], part[(size_t)b * kGfcVals + 4 + k]);
    }
  const double V = (double)e->V;
  double dg[6];
  if (diagnostics_resident(e, dg)) return -1;
  out[0] = 2.0 * sum[0] / (3.0 * V);
  out[1] = mx[0];
  out[2] = 2.0 * sum[1] / (3.0 * V);
  out[3] = mx[1];
  out[4] = dg[4];
  out[5] = dg[5];
  out[6] = 2.0 * sum[2] / (3.0 * V);
  out[7] = mx[2];
  out[8] = 2.0 * sum[3] / (3.0 * V);
  out[9] = mx[3];
  return 0;
}

// latt_reunitU of the links resident in e
template <typename E>
static int reunit_resident(E *e) {
  const size_t nl = (size_t)e->V * 4;
  k_reunit_links<double><<<(unsigned)((nl + 255) / 256), 256, 0, e->s>>>(e->d_U,
                                                                         e->V);
  LAUNCHED(1);
  CK(cudaGetLastError());
  return 0;
}

}  // extern "C++"

int gfix_observables(const double *links, const size_t dims[4], double *out) {
  if (!links || !dims || !out) return fail("null argument");
  Engine<double> *e = engine64(dims);
  if (!e || stage_host(e, links)) return -1;
  return observables_resident(e, out);
}

int gfix_link_diagnostics(const double *links, const size_t dims[4],
                          double *out) {
  if (!links || !dims || !out) return fail("null argument");
  Engine<double> *e = engine64(dims);
  if (!e || stage_host(e, links)) return -1;
  return diagnostics_resident(e, out);
}

int gfix_gf_check(const double *links, const size_t dims[4], double *out) {
  if (!links || !dims || !out) return fail("null argument");
  Engine<double> *e = engine64(dims);
  if (!e || stage_host(e, links)) return -1;
  return gf_check_resident(e, out);
}

int gfix_reunit(double *links, const size_t dims[4]) {
  if (!links || !dims) return fail("null argument");
  Engine<double> *e = engine64(dims);
  if (!e || stage_host(e, links)) return -1;
  const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
  if (reunit_resident(e)) return -1;
  if (e->to_aos(e->d_aos)) return -1;
  CK(cudaMemcpyAsync(links, e->d_aos, bytes, cudaMemcpyDeviceToHost, e->s));
  CK(cudaStreamSynchronize(e->s));
  return 0;
}

int gfix_fourier_accelerate(double *fields, const size_t dims[4], int ndim) {
  if (!fields || !dims) return fail("null argument");
  if (ndim == 3) {
    // one slice: the Coulomb engine of a 2-slice lattice, slice 0 carrying
    // the fields, slice 1 zero (the slices are transformed independently)
    const size_t d3[4] = {dims[0], dims[1], dims[2], 2};
    Engine<double> *e = engine_coul(d3);
    if (!e) return -1;
    Params p;
    if (e->reset(p)) return -1;
    if (e->d_cmask) CK(cudaMemsetAsync(e->d_cmask, 0, 2 * sizeof(int), e->s));
    const size_t lcu = (size_t)e->Lcu, V = (size_t)e->V;
    CK(cudaMemsetAsync(e->c.fb[0], 0, V * 4 * sizeof(cx<double>), e->s));
    for (int k = 0; k < 4; k++)
      CK(cudaMemcpyAsync(e->c.fb[0] + k * V, fields + k * lcu * 2,
                         lcu * sizeof(cx<double>), cudaMemcpyHostToDevice, e->s));
    e->fft(false);
    for (int k = 0; k < 4; k++)
      CK(cudaMemcpyAsync(fields + k * lcu * 2, e->c.fb[0] + k * V,
                         lcu * sizeof(cx<double>), cudaMemcpyDeviceToHost, e->s));
    CK(cudaStreamSynchronize(e->s));
    return 0;
  }
  if (ndim != 4) return fail("ndim %d: the transform is 3 (Coulomb) or 4 (Landau)", ndim);
  Engine<double> *e = engine64(dims);
  if (!e) return -1;
  const size_t bytes = (size_t)e->V * 4 * sizeof(double2);
  Params p;
  if (e->reset(p)) return -1;
  CK(cudaMemcpyAsync(e->c.fb[0], fields, bytes, cudaMemcpyHostToDevice, e->s));
  e->fft(false);
  CK(cudaMemcpyAsync(fields, e->c.fb[0], bytes, cudaMemcpyDeviceToHost, e->s));
  CK(cudaStreamSynchronize(e->s));
  return 0;
}

int gfix_profile_landau(const double *d_links, const size_t dims[4],
                        const gfix_params *p, int iters, double *ms,
                        double *bytes) {
  if (!p) return fail("null params");
  gfix_params pc = *p;  // GFIX_PROFILE_POLISH is a profiling-only value
  if (pc.precision == GFIX_PROFILE_POLISH) pc.precision = GFIX_MIXED;
  if (check_params(dims, &pc)) return -1;
  if (!d_links || !ms || iters < 1) return fail("bad profile arguments");
  Engine<double> *e = engine64(dims);
  if (!e) return -1;
  const size_t n = (size_t)e->V * 36 * sizeof(double2);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpyAsync(e->d_aos, d_links, n, cudaMemcpyDeviceToDevice, e->s));
  if (e->from_aos(e->d_aos)) return -1;
  Params q = to_params(p);
  q.traj_cap = 0;
  if (p->precision == GFIX_PROFILE_POLISH) {
    // the second phase of a mixed solve: FP64 links, FP32 fields
    Engine<double, float> *m = engine64m(dims);
    if (!m) return -1;
    CK(cudaMemcpyAsync(m->d_aos, d_links, n, cudaMemcpyDeviceToDevice, m->s));
    if (m->from_aos(m->d_aos)) return -1;
    return m->profile_cg(q, iters, ms, bytes);
  }
  if (p->precision == GFIX_MIXED) {
    Engine<float> *f = engine32(dims);
    if (!f) return -1;
    CK(cudaStreamSynchronize(e->s));
    k_convert<double, float><<<1184, 256, 0, f->s>>>(e->d_U, f->d_U,
                                                     (size_t)e->V * 4 * kLinkCx);
    k_identity<float><<<(e->V + 255) / 256, 256, 0, f->s>>>(f->d_G, e->V);
    LAUNCHED(2);
    return f->profile_cg(q, iters, ms, bytes);
  }
  return e->profile_cg(q, iters, ms, bytes);
}

// the staged links of `e` (AoS FP64 in e->d_aos) Coulomb-fixed in place.
// GFIX_MIXED: every slice first runs in FP32 (links, g, fields; probes and
// reductions in FP64 arithmetic) to theta < switch_theta, then g is
// widened, reunitarised in FP64 and the FP64 solve continues from it to the
// requested accuracy; a non-finite FP32 phase hands over nothing (FP64 from
// g = 1).  Trajectories then hold the FP64 phase.
static int coulomb_staged(Engine<double> *e, const gfix_params *gp,
                          gfix_result *r, double *slice_theta,
                          size_t *slice_iters, int transform = 1) {
  const Params p = to_params(gp);
  const int T = e->c.L[3];
  std::vector<double> th(T), th32(T);
  std::vector<size_t> it(T), it32(T, 0);
  gfix_result res;
  memset(&res, 0, sizeof res);
  CK(cudaEventRecord(e->ev0, e->s));
  if (e->from_aos(e->d_aos)) return -1;
  size_t iters = 0, tl = 0, n32 = 0;
  bool from_g = false;
  if (gp->precision == GFIX_MIXED) {
    Engine<float> *f = engine_coul32(e->dims);
    if (!f) return -1;
    CK(cudaStreamSynchronize(e->s));
    k_convert<double, float><<<1184, 256, 0, f->s>>>(e->d_U, f->d_U,
                                                     (size_t)e->V * 4 * kLinkCx);
    LAUNCHED(1);
    Params p32 = p;
    p32.acc = gp->switch_theta;
    p32.traj_cap = 0;
    p32.traj_theta = p32.traj_func = nullptr;
    stall_rule(p32);  // per slice (FACG)
    if (f->csolve(p32, &n32, th32.data(), it32.data(), nullptr, true, 0))
      return -1;
    bool finite = true;
    for (int t = 0; t < T; t++) finite &= std::isfinite(th32[t]) != 0;
    if (finite) {
      k_convert<float, double><<<1184, 256, 0, f->s>>>(f->d_G, e->d_G,
                                                       (size_t)e->V * 9);
      LAUNCHED(1);
      CK(cudaStreamSynchronize(f->s));
      k_reunit_mats<double><<<(e->V + 255) / 256, 256, 0, e->s>>>(
          e->d_G, (size_t)e->V);
      LAUNCHED(1);
      from_g = true;
    } else {
      std::fill(it32.begin(), it32.end(), 0);
      n32 = 0;
      res.restarts++;
    }
  }
  if (e->csolve(p, &iters, th.data(), it.data(), &tl, !from_g, transform))
    return -1;
  CK(cudaEventRecord(e->ev1, e->s));
  if (e->to_aos(e->d_aos)) return -1;
  CK(cudaStreamSynchronize(e->s));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
  double worst = 0.0;
  int restarts = res.restarts;
  for (int t = 0; t < T; t++) {
    worst = std::isnan(th[t]) || th[t] > worst ? th[t] : worst;
    restarts += e->h_sl[t].control;
    if (slice_theta) slice_theta[t] = th[t];
    if (slice_iters) slice_iters[t] = it[t] + it32[t];
  }
  res.iters = iters + n32;
  res.iters_fp32 = n32;
  res.theta = worst;
  res.traj_len = tl;
  res.gpu_ms = ms;
  res.restarts = restarts;
  if (r) *r = res;
  return 0;
}

int gfix_coulomb(double *links, const size_t dims[4], const gfix_params *p,
                 gfix_result *r, double *slice_theta, size_t *slice_iters) {
  if (check_params(dims, p)) return -1;
  if (!links) return fail("null links");
  HostArray io(links);
  return gfix::coulomb_io(io, dims, p, r, slice_theta, slice_iters);
}

// (the host-array forms of gfix::landau_driver_io and coulomb_driver_io)
int gfix_landau_driver(double *links, const size_t dims[4], const gfix_params *p,
                       gfix_result *r, double *obs, double *diag) {
  if (check_params(dims, p)) return -1;
  if (!links) return fail("null links");
  HostArray io(links);
  return gfix::landau_driver_io(io, dims, p, r, obs, diag);
}

int gfix_coulomb_driver(double *links, const size_t dims[4], const gfix_params *p,
                        gfix_result *r, double *obs_in, double *diag_in,
                        double *obs, double *diag) {
  if (check_params(dims, p)) return -1;
  if (!links) return fail("null links");
  HostArray io(links);
  return gfix::coulomb_driver_io(io, dims, p, r, obs_in, diag_in, obs, diag);
}

int gfix_profile_coulomb(const double *d_links, const size_t dims[4],
                         const gfix_params *p, int iters, double *ms,
                         double *bytes) {
  if (check_params(dims, p)) return -1;
  if (!d_links || !ms || iters < 1) return fail("bad profile arguments");
  Engine<double> *e = engine_coul(dims);
  if (!e) return -1;
  const size_t n = (size_t)e->V * 36 * sizeof(double2);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpyAsync(e->d_aos, d_links, n, cudaMemcpyDeviceToDevice, e->s));
  if (e->from_aos(e->d_aos)) return -1;
  if (p->precision == GFIX_MIXED) {
    Engine<float> *f = engine_coul32(dims);
    if (!f) return -1;
    CK(cudaStreamSynchronize(e->s));
    k_convert<double, float><<<1184, 256, 0, f->s>>>(e->d_U, f->d_U,
                                                     (size_t)e->V * 4 * kLinkCx);
    LAUNCHED(1);
    return f->profile_coul(to_params(p), iters, ms, bytes);
  }
  return e->profile_coul(to_params(p), iters, ms, bytes);
}

int gfix_coulomb_slices(double *d_links, const size_t dims[4],
                        const gfix_params *p, gfix_result *r,
                        double *slice_theta, size_t *slice_iters,
                        double *d_g_first, double *d_g_last) {
  if (check_params(dims, p)) return -1;
  if (!d_links || !d_g_first || !d_g_last) return fail("null links or g buffer");
  Engine<double> *e = engine_coul(dims);
  if (!e) return -1;
  const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpyAsync(e->d_aos, d_links, bytes, cudaMemcpyDeviceToDevice, e->s));
  if (coulomb_staged(e, p, r, slice_theta, slice_iters, 2)) return -1;
  CK(cudaMemcpyAsync(d_links, e->d_aos, bytes, cudaMemcpyDeviceToDevice, e->s));
  const unsigned nb = (unsigned)((e->Lcu + 127) / 128);
  k_cexport_slice<<<nb, 128, 0, e->s>>>(e->d_G, reinterpret_cast<double2 *>(d_g_first),
                                       e->V, e->Lcu, 0);
  k_cexport_slice<<<nb, 128, 0, e->s>>>(e->d_G, reinterpret_cast<double2 *>(d_g_last),
                                       e->V, e->Lcu, e->c.L[3] - 1);
  LAUNCHED(2);
  CK(cudaStreamSynchronize(e->s));
  return 0;
}

int gfix_coulomb_slices_finish(double *d_links, const size_t dims[4],
                               const double *d_g_last, const double *d_g_next) {
  if (!d_links || !d_g_last || !d_g_next || !dims) return fail("null argument");
  for (int i = 0; i < 4; i++)
    if (dims[i] < 2) return fail("extent %zu of dimension %d below 2", dims[i], i);
  const size_t lcu = dims[0] * dims[1] * dims[2], V = lcu * dims[3];
  if (V > (size_t)INT32_MAX / 4) return fail("lattice volume %zu too large", V);
  CK(cudaDeviceSynchronize());
  k_cfinish_aos<<<(unsigned)((lcu + 127) / 128), 128>>>(
      reinterpret_cast<double2 *>(d_links), reinterpret_cast<const double2 *>(d_g_last),
      reinterpret_cast<const double2 *>(d_g_next), (int)V, (int)lcu);
  LAUNCHED(1);
  CK(cudaDeviceSynchronize());
  return 0;
}

int gfix_coulomb_device(double *d_links, const size_t dims[4],
                        const gfix_params *p, gfix_result *r,
                        double *slice_theta, size_t *slice_iters) {
  if (check_params(dims, p)) return -1;
  if (!d_links) return fail("null links");
  Engine<double> *e = engine_coul(dims);
  if (!e) return -1;
  const size_t bytes = (size_t)e->V * 36 * sizeof(double2);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpyAsync(e->d_aos, d_links, bytes, cudaMemcpyDeviceToDevice, e->s));
  if (coulomb_staged(e, p, r, slice_theta, slice_iters)) return -1;
  CK(cudaMemcpyAsync(d_links, e->d_aos, bytes, cudaMemcpyDeviceToDevice, e->s));
  CK(cudaStreamSynchronize(e->s));
  return 0;
}

struct gfix_batch {
  gfix::Batch b;
};

gfix_batch *gfix_batch_create(const gfix_params *p) {
  if (!p) {
    fail("null params");
    return nullptr;
  }
  if (p->algo != GFIX_CG && p->algo != GFIX_SD) {
    fail("unknown algo %d", p->algo);
    return nullptr;
  }
  if (p->precision != GFIX_FP64 && p->precision != GFIX_MIXED) {
    fail("unknown precision %d", p->precision);
    return nullptr;
  }
  auto *b = new gfix_batch();
  b->b.p = *p;
  b->b.p.traj_theta = b->b.p.traj_func = nullptr;
  b->b.p.traj_cap = 0;
  return b;
}

static int batch_add(gfix_batch *b, double *links, const size_t dims[4],
                     bool device) {
  if (!b || !links) return fail("null batch or links");
  if (check_params(dims, &b->b.p)) return -1;
  auto I = std::make_unique<gfix::BatchInst>();
  for (int k = 0; k < 4; k++) I->dims[k] = dims[k];
  I->links = links;
  I->device = device;
  if (b->b.p.precision == GFIX_MIXED) {
    I->e64m = std::make_unique<Engine<double, float>>();
    if (I->e64m->init(dims, false, true)) return -1;
  } else {
    I->e64 = std::make_unique<Engine<double>>();
    if (I->e64->init(dims, false, true)) return -1;
  }
  b->b.inst.push_back(std::move(I));
  return (int)b->b.inst.size() - 1;
}

int gfix_batch_add(gfix_batch *b, double *links, const size_t dims[4]) {
  return batch_add(b, links, dims, false);
}

int gfix_batch_add_device(gfix_batch *b, double *d_links, const size_t dims[4]) {
  return batch_add(b, d_links, dims, true);
}

int gfix_batch_run(gfix_batch *b) {
  if (!b) return fail("null batch");
  return gfix::batch_run(&b->b);
}

int gfix_batch_result(const gfix_batch *b, int i, gfix_result *r) {
  if (!b || !r || i < 0 || (size_t)i >= b->b.inst.size())
    return fail("no configuration %d in the batch", i);
  *r = b->b.inst[(size_t)i]->res;
  return 0;
}

void gfix_batch_destroy(gfix_batch *b) { delete b; }

}  // extern "C"

// ---------------------------------------------------------------------
// the solves with the links moved by a LinkIO (the flat host entry points
// above, and GLU's own entry points)

namespace gfix {

int landau_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
              gfix_result *r) {
  if (check_params(dims, p)) return -1;
  return with_landau_engine(dims, p->precision, [&](auto *e) -> int {
    // (a mixed solve's FP32 engine is made here too, not inside the solve)
    if (p->precision == GFIX_MIXED && !engine32(dims)) return -1;
    if (mark(e->s, "engine") || io.to_device(e->d_aos, e->V, e->s) ||
        mark(e->s, "to device"))
      return -1;
    if (landau_staged(e, p, r) || mark(e->s, "solve")) return -1;
    return (io.to_host(e->d_aos, e->V, e->s) || mark(e->s, "to host")) ? -1 : 0;
  });
}

// GLU's Landau driver in one device-resident sequence: the solve with its
// random restarts, then -- when it converged -- output_fixing_info's
// reunitarisation and diagnostics, all on the links in HBM, so the links
// cross PCIe once each way.
int landau_driver_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
                     gfix_result *r, double *obs, double *diag) {
  if (check_params(dims, p)) return -1;
  return with_landau_engine(dims, p->precision, [&](auto *e) -> int {
    if (p->precision == GFIX_MIXED && !engine32(dims)) return -1;
    if (mark(e->s, "engine") || io.to_device(e->d_aos, e->V, e->s) ||
        mark(e->s, "to device"))
      return -1;
    gfix_result res;
    if (landau_staged(e, p, &res) || mark(e->s, "solve")) return -1;
    if (res.iters != kSentinel && res.iters != kGluFailure) {
      if (reunit_resident(e)) return -1;
      if (obs && observables_resident(e, obs)) return -1;
      if (diag && diagnostics_resident(e, diag)) return -1;
      if (e->to_aos(e->d_aos)) return -1;
    } else {
      if (obs) memset(obs, 0, 3 * sizeof(double));
      if (diag) memset(diag, 0, 6 * sizeof(double));
    }
    if (mark(e->s, "post") || io.to_host(e->d_aos, e->V, e->s) ||
        mark(e->s, "to host"))
      return -1;
    if (r) *r = res;
    return 0;
  });
}

int coulomb_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
               gfix_result *r, double *slice_theta, size_t *slice_iters) {
  if (check_params(dims, p)) return -1;
  Engine<double> *e = engine_coul(dims);
  if (!e || mark(e->s, "engine") || io.to_device(e->d_aos, e->V, e->s) ||
      mark(e->s, "to device"))
    return -1;
  if (coulomb_staged(e, p, r, slice_theta, slice_iters) || mark(e->s, "solve"))
    return -1;
  return (io.to_host(e->d_aos, e->V, e->s) || mark(e->s, "to host")) ? -1 : 0;
}

// GLU's Coulomb driver in one device-resident sequence: the diagnostics of
// the input, the solve of every slice with the slice transforms, the final
// reunitarisation and the diagnostics of the result.
int coulomb_driver_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
                      gfix_result *r, double *obs_in, double *diag_in,
                      double *obs, double *diag) {
  if (check_params(dims, p)) return -1;
  Engine<double> *e = engine_coul(dims);
  if (!e || mark(e->s, "engine") || io.to_device(e->d_aos, e->V, e->s) ||
      mark(e->s, "to device"))
    return -1;
  if (obs_in || diag_in) {
    if (e->from_aos(e->d_aos)) return -1;
    if (obs_in && observables_resident(e, obs_in)) return -1;
    if (diag_in && diagnostics_resident(e, diag_in)) return -1;
  }
  gfix_result res;
  if (coulomb_staged(e, p, &res, nullptr, nullptr) || mark(e->s, "solve")) return -1;
  if (reunit_resident(e)) return -1;
  if (obs && observables_resident(e, obs)) return -1;
  if (diag && diagnostics_resident(e, diag)) return -1;
  if (e->to_aos(e->d_aos) || mark(e->s, "post")) return -1;
  if (io.to_host(e->d_aos, e->V, e->s) || mark(e->s, "to host")) return -1;
  if (r) *r = res;
  return 0;
}

}  // namespace gfix
