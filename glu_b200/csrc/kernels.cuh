// Device kernels of the Fourier-accelerated Landau gauge fixing on B200.
//
// One iteration of FACG (src/Gfix/FACG.c:270-334) is the launch sequence
//   k_deriv          Delta(x) packed in 4 fields + theta and Re tr U partials
//   k_scalar THETA   theta, functional, stop decision
//   k_fft_xy  fwd    x,y passes of the 4D FFT, one xy-plane per block
//   k_fft_zt         z,t passes, * psq, inverse t,z passes (one tile/block)
//   k_fft_xy  bwd    inverse x,y passes fused with the PR sums
//   k_scalar PR      beta (PR+ / FR switch at CG_TOL)
//   k_dir_probe      sn <- in + beta sn, line-search probes of GLU's
//                    line_search_Landau (src/Gfix/line_search.c:274-341)
//   k_scalar PROBES  alpha* by the parabola of approx_minimum
//   k_update         U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag, g = reunit(1+a A)
//   k_scalar END     iteration count, buffer parities, done flag
// Every kernel first checks the device-side done flag, so a captured graph
// of the iteration can be replayed past convergence as a no-op.
//
// HBM layout (SoA, site index s = x + Lx (y + Ly (z + Lz t))):
//   U   cx<R>[4 mu][6 elements][V]        links: their first two columns
//                                          (load_link rebuilds the third)
//   fb  cx<F>[2][4 fields][V]             in / in_old (parity selects)
//   sb  cx<F>[2][4 fields][V]             sn ping-pong (sparity selects)
//   G   cx<R>[9][V]                        accumulated gauge transform
//                                          (mixed precision only)
// R is the type of the links (and of the link arithmetic), F that of the
// su(3) fields and of the FFT: F = R except in the FP64 phase of a
// mixed-precision solve, which keeps FP64 links, theta and updates but
// carries its search directions and their Fourier acceleration in FP32.
#pragma once

#include "fft.cuh"
#include "su3.cuh"

namespace gfix {

constexpr double kCgTol = 5E-11;            // GLU_definitions.h:451-455
constexpr double kVal49 = 0.4444444444444444;  // lin_derivs.c:72
constexpr int kSiteThreads = 128;
constexpr int kScalarThreads = 1024;

enum ScalarOp : int {
  OP_THETA_TEST = 0,  // theta_test_lin = 2 sum / (NC V)
  OP_THETA_SD,        // theta of an SD start: reduction slots carry over
  OP_THETA_MAIN,      // theta at the top of a CG/SD iteration
  OP_PR,              // beta of the CG direction
  OP_PROBES,          // alpha* from the probes (or the fixed step)
  OP_DER,             // inold after the SD start
  OP_END_CG,          // end of a CG iteration
  OP_END_SD,          // end of an SD (FASD) iteration
  OP_ALPHA_FIXED,     // step = gf_alpha (SD without line search)
};

struct DevState {
  double tr;          // in-loop theta of the current iteration
  double tr_test;     // theta_test_lin
  double func;        // gauge functional of the current links
  double inold, insum, sumconj, beta, alpha;
  double ls_last[2];  // probe sums left in GLU's reduction slots
  double insum_last;  // insum left in GLU's reduction slot
  double gf_alpha, acc;
  long long max_iters;
  long long iter;     // loc_iters of the current run
  long long traj_len, traj_cap;
  double *traj_theta, *traj_func;
  int use_ls;         // this step uses the line search
  int stop;           // current iteration is the last one of the run
  int done;           // run finished: kernels return at once
  int parity;         // fb[parity] = in, fb[parity ^ 1] = in_old
  int sparity;        // sb[sparity] = sn (old), sb[sparity ^ 1] = new
  int nblocks;        // partials written by the last reduction kernel
  int sd_fixed;       // GLU_GFIX_SD: fixed step gf_alpha in SD steps
  double cg_tol;      // CG_TOL (GLU_definitions.h:451-455)
  double hp_below;    // FP32 storage: probes in FP64 arithmetic once tr < this
  // stall rule of a mixed-precision FP32 phase (stall_window 0: off): once
  // the best theta is below stall_floor, the run ends when theta has not
  // improved on it by 10% for stall_window iterations or exceeds blowup x it
  double best_tr, stall_floor, blowup;
  long long since_best, stall_window;
};

// which arithmetic variant of a kernel runs this step (FP32 storage: FP32
// arithmetic while theta >= hp_below, FP64 arithmetic below; a NaN theta
// takes the FP32 variant)
enum ArithSel : int { SEL_ALWAYS = 0, SEL_LOW = 1, SEL_HIGH = 2 };
__device__ __forceinline__ bool arith_skip(int sel, double tr, double below) {
  const bool high = tr < below;
  return (sel == SEL_LOW && high) || (sel == SEL_HIGH && !high);
}

// set or clear the done flag (used to run every kernel once as a no-op)
__global__ void k_set_done(DevState *st, int v) { st->done = v; }

// start of a solver run (GLU's steep_Landau_FACG / _FASD entry)
__global__ void k_begin_run(DevState *st) {
  st->iter = 0;
  st->done = 0;
  st->stop = 0;
  st->use_ls = !st->sd_fixed;
}

template <typename R, typename F = R>
struct Ctx {
  cx<R> *U;
  cx<F> *fb[2];
  cx<F> *sb[2];
  cx<R> *G;
  DevState *st;
  double *part;       // [nblocks][2] per-block partial sums
  const cx<F> *tw;    // twiddle pool
  const double *cs;   // cos tables, cs[mu * cs_ld + n] = cos(n 2pi/L_mu)
  int cs_ld;
  int L[4];
  int V;
  int ndim;           // FFT rank: 4 Landau, 3 Coulomb
  int zt_b;           // x columns per zt tile
  int xy_pitch;       // padded row pitch of the xy tile
  double maxp;        // MAX_LANDAU = 4 ND / V or MAX_COULOMB = 4 (ND-1)/Lcu
  FftAxis ax[4];
  const int *skip;    // ndim 3: per-slice flags, set slices are not transformed
};

// ---------------------------------------------------------------------
// helpers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum of NV values; thread 0 writes them to out[0..NV)
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double *out) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) sh[k][warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double x = lane < nw ? sh[k][lane] : 0.0;
      x = warp_sum(x);
      if (lane == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ void coords(int s, const int *L, int *x) {
  x[0] = s % L[0];
  s /= L[0];
  x[1] = s % L[1];
  s /= L[1];
  x[2] = s % L[2];
  x[3] = s / L[2];
}

__device__ __forceinline__ int fwd_site(int s, int mu, const int *x,
                                        const int *L, const int *stride) {
  return x[mu] == L[mu] - 1 ? s - (L[mu] - 1) * stride[mu] : s + stride[mu];
}
__device__ __forceinline__ int bck_site(int s, int mu, const int *x,
                                        const int *L, const int *stride) {
  return x[mu] == 0 ? s + (L[mu] - 1) * stride[mu] : s - stride[mu];
}

template <typename CT>
__device__ __forceinline__ void strides(const CT &c, int *st) {
  st[0] = 1;
  st[1] = c.L[0];
  st[2] = c.L[0] * c.L[1];
  st[3] = c.L[0] * c.L[1] * c.L[2];
}

// Links in HBM keep their first two columns only: the complex entries
// 0, 1, 3, 4, 6, 7 of the row-major matrix, stored U[mu][k][V], k = 0..5
// (96 of a link's 144 bytes in FP64).  The third column is rebuilt on every
// load as the conjugate cross product of the first two -- the expression
// with which GLU's update (gtransform, src/Gfix/gtrans.c:107-121) and this
// library's own (su3.cuh) complete every link they write -- so a link that
// has been updated once reads back bit for bit as it was computed, and an
// SU(3) input differs from its stored third column by rounding only.
constexpr int kLinkCx = 6;

template <typename R>
__device__ __forceinline__ void load_link(const cx<R> *U, int V, int mu, int s,
                                          cx<R> *u) {
  const cx<R> *p = U + (size_t)mu * kLinkCx * V + s;
  u[0] = p[0];
  u[1] = p[(size_t)V];
  u[3] = p[2 * (size_t)V];
  u[4] = p[3 * (size_t)V];
  u[6] = p[4 * (size_t)V];
  u[7] = p[5 * (size_t)V];
  complete_col2(u);
}

template <typename R>
__device__ __forceinline__ void store_link(cx<R> *U, int V, int mu, int s,
                                           const cx<R> *u) {
  cx<R> *p = U + (size_t)mu * kLinkCx * V + s;
  p[0] = u[0];
  p[(size_t)V] = u[1];
  p[2 * (size_t)V] = u[3];
  p[3 * (size_t)V] = u[4];
  p[4 * (size_t)V] = u[6];
  p[5 * (size_t)V] = u[7];
}

// ---------------------------------------------------------------------
// K1: the gauge derivative, fused with the theta and functional sums
// (src/Gfix/lin_derivs.c:74-193 packed as src/Gfix/FACG.c:54-60)

template <typename R, typename F = R>
__global__ void __launch_bounds__(kSiteThreads)
    k_deriv(Ctx<R, F> c) {
  if (c.st->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (s < c.V) {
    int x[4], sd[4];
    coords(s, c.L, x);
    strides(c, sd);
    R R0 = 0, R1 = 0, I1 = 0, R2 = 0, I2 = 0, R3 = 0, R4 = 0, I4 = 0;
    double re = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      cx<R> q[9], b[9];
      load_link(c.U, c.V, mu, s, q);
      load_link(c.U, c.V, mu, bck_site(s, mu, x, c.L, sd), b);
      const cx<R> q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4],
                  q5 = q[5], q6 = q[6], q7 = q[7], q8 = q[8];
      const cx<R> b0 = b[0], b1 = b[1], b2 = b[2], b3 = b[3], b4 = b[4],
                  b5 = b[5], b6 = b[6], b7 = b[7], b8 = b[8];
      R0 += R(2) * b0.y - b4.y - b8.y;
      R0 += R(-2) * q0.y + q4.y + q8.y;
      R1 += b1.x - b3.x - q1.x + q3.x;
      I1 += b1.y + b3.y - q1.y - q3.y;
      R2 += b2.x - b6.x - q2.x + q6.x;
      I2 += b2.y + b6.y - q2.y - q6.y;
      R3 += R(2) * b4.y - b0.y - b8.y;
      R3 += R(-2) * q4.y + q0.y + q8.y;
      R4 += b5.x - b7.x - q5.x + q7.x;
      I4 += b5.y + b7.y - q5.y - q7.y;
      re += (double)q0.x + (double)q4.x + (double)q8.x;
    }
    cx<F> *f = c.fb[c.st->parity];
    const size_t V = c.V;
    f[s] = mk<F>((F)(-(R3 / R(3))), (F)(R0 / R(3)));
    f[V + s] = mk<F>((F)(R(0.5) * R1), (F)(R(0.5) * I1));
    f[2 * V + s] = mk<F>((F)(R(0.5) * R2), (F)(R(0.5) * I2));
    f[3 * V + s] = mk<F>((F)(R(0.5) * R4), (F)(R(0.5) * I4));
    const double d0 = R0, d1 = R1, e1 = I1, d2 = R2, e2 = I2, d3 = R3,
                 d4 = R4, e4 = I4;
    v[0] = kVal49 * (d0 * d0 + d3 * (d3 + d0)) +
           (d1 * d1 + e1 * e1 + d2 * d2 + e2 * e2 + d4 * d4 + e4 * e4);
    v[1] = re;
  }
  block_sum_store<2>(v, c.part + 2 * blockIdx.x);
  if (threadIdx.x == 0 && blockIdx.x == 0) c.st->nblocks = gridDim.x;
}

// ---------------------------------------------------------------------
// the 4D (or batched 3D) FFT with psq folded into the middle pass

#include "fft_pass.cuh"
#include "fft_ct.cuh"

// ---------------------------------------------------------------------
// K4: conjugate direction update fused with the line-search probes.
// DIR: sn_new = in + beta sn_old (src/Gfix/FACG.c:315-323), else the
// direction is `in` itself (an SD step).  Probes: per site the three
// values of src/Gfix/line_search.c:296-313 at alpha = 0, 0.15, 0.30;
// accumulated as differences to the alpha = 0 value, which leaves the
// parabola of approx_minimum unchanged and avoids cancelling large sums.

// the direction at site s as stored (type F): computed in R, rounded to F;
// f receives it back in R, so the probes use the direction the update reads
template <typename R, bool DIR, typename F>
__device__ __forceinline__ void dir_at(const Ctx<R, F> &c, const cx<F> *in,
                                       const cx<F> *so, R beta, int s,
                                       cx<R> *f, cx<F> *fs = nullptr) {
  const size_t V = c.V;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const cx<F> a = in[k * V + s];
    cx<F> r;
    if (DIR) {
      const cx<F> b = so[k * V + s];
      r = mk<F>((F)fma(beta, (R)b.x, (R)a.x), (F)fma(beta, (R)b.y, (R)a.y));
    } else {
      r = a;
    }
    if (fs) fs[k] = r;
    f[k] = mk<R>((R)r.x, (R)r.y);
  }
}

// C is the arithmetic precision of the probes: the FP32 phase of the mixed
// solver evaluates them in FP64 from its FP32 links and directions once
// theta < hp_below (1e-5), because per-site probe differences fall below
// FP32 rounding once theta < ~1e-6; above it FP32 arithmetic serves.  Both
// variants are launched, `sel` lets the one that fits the step run.
template <typename R, bool DIR, typename C = R, typename F = R>
__global__ void __launch_bounds__(kSiteThreads) k_dir_probe(Ctx<R, F> c, int sel) {
  if (c.st->done || arith_skip(sel, c.st->tr, c.st->hp_below)) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int par = c.st->parity, spar = c.st->sparity;
  const cx<F> *in = c.fb[par];
  const cx<F> *so = c.sb[spar];
  cx<F> *sn = c.sb[spar ^ 1];
  const R beta = (R)c.st->beta;
  const bool probes = c.st->use_ls != 0;
  double v[2] = {0.0, 0.0};
  if (s < c.V) {
    cx<R> f[4];
    cx<F> fs[4];
    dir_at<R, DIR>(c, in, so, beta, s, f, fs);
    if (DIR) {
#pragma unroll
      for (int k = 0; k < 4; k++) sn[(size_t)k * c.V + s] = fs[k];
    }
    if (probes) {
      int x[4], sd[4];
      coords(s, c.L, x);
      strides(c, sd);
      auto up = [](cx<R> a) { return mk<C>((C)a.x, (C)a.y); };
      // one probe at a time: a single matrix at x stays live
      C d[2] = {0, 0};
#pragma unroll 1
      for (int k = 0; k < 2; k++) {
        const C al = k == 0 ? C(0.15) : C(0.30);
        cx<C> A[9], Bm[9], U[9];
        set_gauge(A, up(f[0]), up(f[1]), up(f[2]), up(f[3]), al);
#pragma unroll 1
        for (int mu = 0; mu < 4; mu++) {
          const int y = fwd_site(s, mu, x, c.L, sd);
          cx<R> fy[4];
          dir_at<R, DIR>(c, in, so, beta, y, fy);
          cx<R> u[9];
          load_link(c.U, c.V, mu, s, u);
#pragma unroll
          for (int e = 0; e < 9; e++) U[e] = up(u[e]);
          const C t0 = U[0].x + U[4].x + U[8].x;
          set_gauge(Bm, up(fy[0]), up(fy[1]), up(fy[2]), up(fy[3]), al);
          d[k] += re_tr_abc_dag(A, U, Bm) - t0;
        }
      }
      const C d1 = d[0], d2 = d[1];
      v[0] = d1;
      v[1] = d2;
    }
  }
  if (probes) {
    block_sum_store<2>(v, c.part + 2 * blockIdx.x);
    if (threadIdx.x == 0 && blockIdx.x == 0) c.st->nblocks = gridDim.x;
  }
}

// ---------------------------------------------------------------------
// K5: the link update of egauge_Landau (src/Gfix/line_search.c:60-97):
// g(x) = reunit(1 + alpha A(x)), U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag.
// SN selects the direction: the new conjugate direction or `in`.
// With G (mixed precision) the transform is accumulated, G(x) <- g(x) G(x).

template <typename R, bool SN, typename F = R>
__global__ void __launch_bounds__(kSiteThreads) k_update(Ctx<R, F> c) {
  if (c.st->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.V) return;
  const cx<F> *d = SN ? c.sb[c.st->sparity ^ 1] : c.fb[c.st->parity];
  const R alpha = (R)c.st->alpha;
  const size_t V = c.V;
  int x[4], sd[4];
  coords(s, c.L, x);
  strides(c, sd);
  auto up = [](cx<F> a) { return mk<R>((R)a.x, (R)a.y); };
  cx<R> A[9], Bm[9], U[9];
  set_gauge(A, up(d[s]), up(d[V + s]), up(d[2 * V + s]), up(d[3 * V + s]), alpha);
#pragma unroll 1
  for (int mu = 0; mu < 4; mu++) {
    const int y = fwd_site(s, mu, x, c.L, sd);
    set_gauge(Bm, up(d[y]), up(d[V + y]), up(d[2 * V + y]), up(d[3 * V + y]), alpha);
    load_link(c.U, c.V, mu, s, U);
    gtransform(A, U, Bm);
    store_link(c.U, c.V, mu, s, U);
  }
  if (c.G) {
    cx<R> g[9], r[9];
#pragma unroll
    for (int e = 0; e < 9; e++) g[e] = c.G[(size_t)e * V + s];
    multab(r, A, g);
#pragma unroll
    for (int e = 0; e < 9; e++) c.G[(size_t)e * V + s] = r[e];
  }
}

// sn = in_old = in after an SD start, with sum_DER3 (src/Gfix/FACG.c:148-178)
template <typename R>
__global__ void __launch_bounds__(256) k_copy_der(Ctx<R> c) {
  if (c.st->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const cx<R> *in = c.fb[c.st->parity];
  cx<R> *sn = c.sb[c.st->sparity];
  double v[1] = {0.0};
  if (s < c.V) {
    double l = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const cx<R> a = in[(size_t)k * c.V + s];
      sn[(size_t)k * c.V + s] = a;
      const double ar = a.x, ai = a.y;
      l += (k == 0) ? (ar * ar + ai * ai + ar * ai) : (ar * ar + ai * ai);
    }
    v[0] = 2.0 * l;
  }
  block_sum_store<1>(v, c.part + blockIdx.x);
  if (threadIdx.x == 0 && blockIdx.x == 0) c.st->nblocks = gridDim.x;
}

// ---------------------------------------------------------------------
// scalar logic: one block reduces the partials in a fixed order and applies
// GLU's control flow for the step.

__device__ __forceinline__ double approx_minimum(const double *al,
                                                 const double *f) {
  // src/Gfix/line_search.c:38-57
  const double A = f[0] / ((al[0] - al[1]) * (al[0] - al[2]));
  const double B = f[1] / ((al[1] - al[0]) * (al[1] - al[2]));
  const double C = f[2] / ((al[2] - al[0]) * (al[2] - al[1]));
  const double Sol = (al[0] * (B + C) + al[1] * (A + C) + al[2] * (A + B)) /
                     (2 * (A + B + C));
  if (Sol > al[2]) return al[2];
  if (isnan(Sol) || isinf(Sol) || Sol < al[0]) return 0.08;
  return Sol;
}

__global__ void __launch_bounds__(kScalarThreads)
    k_scalar(DevState *st, const double *part, int op, int nv, double norm_v) {
  if (st->done) return;
  const int nb = st->nblocks;
  double a[2] = {0.0, 0.0};
  if (op != OP_END_CG && op != OP_END_SD && op != OP_ALPHA_FIXED) {
    // eight independent loads in flight per thread and round, then added
    // in a fixed order: the sum is deterministic and pays the L2 latency
    // once per eight partials instead of once per partial
    constexpr int kU = 8;
    const int B = blockDim.x;
    for (int i0 = threadIdx.x; i0 < nb; i0 += kU * B) {
      double x0[kU], x1[kU];
#pragma unroll
      for (int k = 0; k < kU; k++) {
        const int i = i0 + k * B;
        x0[k] = i < nb ? part[(size_t)nv * i] : 0.0;
        x1[k] = (nv > 1 && i < nb) ? part[(size_t)nv * i + 1] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < kU; k++) {
        a[0] += x0[k];
        a[1] += x1[k];
      }
    }
    __shared__ double tot[2];
    block_sum_store<2>(a, tot);
    __syncthreads();
    a[0] = tot[0];
    a[1] = tot[1];
  }
  if (threadIdx.x != 0) return;
  // norm_v = number of sites V
  const double V = norm_v;
  switch (op) {
    case OP_THETA_TEST:
      st->tr_test = 2.0 * a[0] / (3.0 * V);
      st->func = 1.0 - a[1] / (12.0 * V);
      break;
    case OP_THETA_SD:
    case OP_THETA_MAIN: {
      st->tr = a[0] / (3.0 * V);  // GFNORM_LANDAU
      st->func = 1.0 - a[1] / (12.0 * V);
      if (st->traj_theta && st->traj_len < st->traj_cap) {
        st->traj_theta[st->traj_len] = st->tr;
        st->traj_func[st->traj_len] = st->func;
        st->traj_len++;
      }
      if (op == OP_THETA_MAIN) {
        // the top of a loop iteration zeroes GLU's reduction slots
        st->ls_last[0] = st->ls_last[1] = 0.0;
        st->stop = !((st->tr > st->acc) && (st->iter + 1 < st->max_iters));
        if (st->stall_window > 0) {
          if (st->tr < 0.9 * st->best_tr) {
            st->best_tr = st->tr;
            st->since_best = 0;
          } else {
            st->since_best++;
          }
          if (st->best_tr < st->stall_floor &&
              (st->since_best >= st->stall_window || st->tr > st->blowup * st->best_tr))
            st->stop = 1;
        }
      }
      break;
    }
    case OP_PR: {
      st->insum = a[0];
      st->sumconj = a[1];
      const double b = st->sumconj / st->inold;
      double beta = (b < 0.0) ? 0.0 : b;  // PRfmax (src/Gfix/CG.c:37-41)
      if (st->tr < st->cg_tol) beta = st->insum / st->inold;
      st->beta = beta;
      st->inold = st->insum;
      st->insum_last = st->insum;
      st->use_ls = st->tr > st->cg_tol;
      break;
    }
    case OP_PROBES: {
      if (st->use_ls) {
        const double d1 = a[0] + st->ls_last[0], d2 = a[1] + st->ls_last[1];
        st->ls_last[0] = d1;
        st->ls_last[1] = d2;
        const double al[3] = {0.0, 0.15, 0.30};
        const double f[3] = {0.0, -d1, -d2};
        st->alpha = approx_minimum(al, f);
      } else {
        st->alpha = st->gf_alpha;
      }
      break;
    }
    case OP_ALPHA_FIXED:
      st->alpha = st->gf_alpha;
      break;
    case OP_DER:
      st->inold = st->insum_last + a[0];
      st->parity ^= 1;  // in_old = in
      break;
    case OP_END_CG:
      st->iter++;
      st->parity ^= 1;
      st->sparity ^= 1;
      if (st->stop) st->done = 1;
      break;
    case OP_END_SD:
      st->iter++;
      if (st->stop) st->done = 1;
      break;
  }
}

// ---------------------------------------------------------------------
// layout conversion: host AoS double[V][4][9][2] <-> device SoA cx<R>

// One block moves kTrSites consecutive sites through shared memory so that
// both the AoS side (36 contiguous complex numbers per site) and the SoA side
// (kTrSites contiguous numbers per element row) are accessed coalesced.
constexpr int kTrSites = 64;

// matrix entry of stored element k of a link (its first two columns)
__device__ __forceinline__ int stored_entry(int k) { return (k >> 1) * 3 + (k & 1); }

template <typename R>
__global__ void __launch_bounds__(256) k_aos_to_soa(const double *__restrict__ aos,
                                                    cx<R> *U, int V) {
  __shared__ double2 t[kTrSites * 36 + 1];
  const size_t s0 = (size_t)blockIdx.x * kTrSites;
  const int ns = (int)min((size_t)kTrSites, (size_t)V - s0);
  const double2 *src = reinterpret_cast<const double2 *>(aos) + s0 * 36;
  for (int i = threadIdx.x; i < ns * 36; i += blockDim.x) t[i] = src[i];
  __syncthreads();
  // row r of the SoA links: direction r / 6, stored element r % 6
  for (int i = threadIdx.x; i < 4 * kLinkCx * kTrSites; i += blockDim.x) {
    const int r = i / kTrSites, sl = i % kTrSites;
    if (sl < ns) {
      const double2 v = t[sl * 36 + (r / kLinkCx) * 9 + stored_entry(r % kLinkCx)];
      U[(size_t)r * V + s0 + sl] = mk<R>((R)v.x, (R)v.y);
    }
  }
}

// one thread per (site, direction) of the block's kTrSites sites: the link
// completed in R (third column rebuilt as in load_link), then staged in
// shared memory for coalesced AoS stores
template <typename R>
__global__ void __launch_bounds__(256) k_soa_to_aos(const cx<R> *U,
                                                    double *__restrict__ aos,
                                                    int V) {
  __shared__ double2 t[kTrSites * 36 + 1];
  const size_t s0 = (size_t)blockIdx.x * kTrSites;
  const int ns = (int)min((size_t)kTrSites, (size_t)V - s0);
  for (int i = threadIdx.x; i < 4 * kTrSites; i += blockDim.x) {
    const int mu = i / kTrSites, sl = i % kTrSites;
    if (sl < ns) {
      cx<R> u[9];
      load_link(U, V, mu, (int)(s0 + sl), u);
#pragma unroll
      for (int e = 0; e < 9; e++)
        t[sl * 36 + mu * 9 + e] = make_double2((double)u[e].x, (double)u[e].y);
    }
  }
  __syncthreads();
  double2 *dst = reinterpret_cast<double2 *>(aos) + s0 * 36;
  for (int i = threadIdx.x; i < ns * 36; i += blockDim.x) dst[i] = t[i];
}

}  // namespace gfix
