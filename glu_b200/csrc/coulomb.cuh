// Coulomb gauge fixing of every time slice at once (GLU's Coulomb_FA,
// src/Gfix/CFACG.c:531-636, solves the slices one after the other; they are
// independent problems on the original spatial links, so here all of them
// advance together, each with its own scalars, iteration count and end).
//
// Per slice t the unknown is the slice gauge field g_t(x) (SoA [9][V], the
// slices side by side), the derivative is taken on the rotated links
// g(x) U_i(x,t) g(x+i)^dag (steep_deriv_CG, CFACG.c:91-163), the FFT is the
// 3D transform of each slice (FOURIER_ACCELERATE2) done by the Landau passes
// with ndim = 3, and the update is g <- reunit(1 + a A) g
// (exponentiate_gauge_CG, line_search.c:101-115).  Each step of a slice is
// either an SD step (a run's first step, every FASD step) or a CG step.
// A slice whose run ends is reunitarised and checked (adequate_solution,
// CFACG.c:432-456), continued, or restarted from a random g (steep_fix,
// CFACG.c:459-529); finished slices are masked out of every kernel.
#pragma once

#include "kernels.cuh"

namespace gfix {

// PREC_TOL (GLU_definitions.h:359-363): NC 1e-14 in double, NC 1e-6 in
// single precision builds
constexpr double kPrecTol = 3 * 1.0E-14;
constexpr double kPrecTolSingle = 3 * 1.0E-6;
constexpr int kCoulThreads = 128;

enum SliceMode : int { SL_RUN = 0, SL_DONE = 1 };

struct Slice {
  double tr, inold, insum, sumconj, beta, alpha;
  long long iter;     // steps of the current run (GLU's loc_iters)
  long long tot;      // GLU's tot_iters of steep_fix
  int sd;             // next step is an SD step
  int use_ls;
  int mode;           // SL_RUN / SL_DONE
  int control;        // random restarts so far
  int reunit;         // maintenance: reunitarise g_t and check it
  int randomize;      // maintenance: random restart of g_t
  int bad;            // set when the unitarity check fails
  int trans;          // GLU's trans_flag: survives a continuation run
  int traj_len;
  double best_tr;     // stall rule (mixed-precision FP32 phase)
  long long since_best;
};

struct CoulState {
  double gf_alpha, acc, cg_tol;
  long long max_iters;
  int facg;           // 1 FACG, 0 FASD
  int sd_fixed;       // GLU_GFIX_SD semantics
  int active;         // slices still running
  int nslices;
  unsigned long long seed;
  int traj_cap;       // per slice
  double *traj;       // [nslices][traj_cap]
  int *done_mask;     // [nslices], 1 once a slice has finished (FFT passes skip it)
  double prec_tol;    // PREC_TOL of the unitarity check
  double hp_below;    // FP32 storage: FP64 arithmetic for slices below this theta
  // stall rule of a mixed-precision FP32 phase (stall_window 0: off): a
  // slice whose best theta is below stall_floor ends its run after
  // stall_window iterations without a 10% improvement on it, or on a jump
  // above blowup x it; the FP64 phase then continues it
  long long stall_window;
  double stall_floor, blowup;
};

template <typename R>
struct CCtx {
  cx<R> *U;           // links SoA [4][9][V]
  cx<R> *g;           // slice gauge fields SoA [9][V]
  cx<R> *fb[2];       // in / in_old
  cx<R> *sb[2];       // sn ping-pong
  DevState *st;       // parities (shared with the FFT passes)
  CoulState *cs;
  Slice *sl;
  double *part;       // [nslices][nbs][2]
  int L[4];
  int V, Lcu, nbs;
};

// slice-site coordinates and the in-slice neighbours of site i in direction
// MU (compile-time, so no index array lands in local memory)
struct SliceSite {
  int i, x[3];
};
__device__ __forceinline__ SliceSite slice_site(int i, const int *L) {
  SliceSite q;
  q.i = i;
  q.x[0] = i % L[0];
  const int r = i / L[0];
  q.x[1] = r % L[1];
  q.x[2] = r / L[1];
  return q;
}
template <int MU>
__device__ __forceinline__ int sfwd(const SliceSite &q, const int *L) {
  const int sd = MU == 0 ? 1 : MU == 1 ? L[0] : L[0] * L[1];
  return q.x[MU] == L[MU] - 1 ? q.i - (L[MU] - 1) * sd : q.i + sd;
}
// the same with a run-time direction, by selects
__device__ __forceinline__ int sfwd_rt(const SliceSite &q, const int *L, int mu) {
  const int xm = mu == 0 ? q.x[0] : mu == 1 ? q.x[1] : q.x[2];
  const int lm = mu == 0 ? L[0] : mu == 1 ? L[1] : L[2];
  const int sd = mu == 0 ? 1 : mu == 1 ? L[0] : L[0] * L[1];
  return xm == lm - 1 ? q.i - (lm - 1) * sd : q.i + sd;
}
template <int MU>
__device__ __forceinline__ int sbck(const SliceSite &q, const int *L) {
  const int sd = MU == 0 ? 1 : MU == 1 ? L[0] : L[0] * L[1];
  return q.x[MU] == 0 ? q.i + (L[MU] - 1) * sd : q.i - sd;
}

// buffer of a ping-pong pair by parity, as a select (a runtime index into
// the by-value kernel parameter would copy it to local memory)
template <typename T>
__device__ __forceinline__ T *pick(T *const (&b)[2], int p) {
  return p ? b[1] : b[0];
}

template <typename R>
__device__ __forceinline__ void load9(const cx<R> *p, int V, int s, cx<R> *u) {
#pragma unroll
  for (int e = 0; e < 9; e++) u[e] = p[(size_t)e * V + s];
}
template <typename R>
__device__ __forceinline__ void store9(cx<R> *p, int V, int s, const cx<R> *u) {
#pragma unroll
  for (int e = 0; e < 9; e++) p[(size_t)e * V + s] = u[e];
}

// rotated link g(a) U g(b)^dag of the reference's gtransform_local
template <typename R>
__device__ __forceinline__ void rotated(const CCtx<R> &c, int mu, int s_link,
                                        int sa, int sb, cx<R> *C) {
  cx<R> A[9], B[9];
  load_link(c.U, c.V, mu, s_link, C);
  load9(c.g, c.V, sa, A);
  load9(c.g, c.V, sb, B);
  gtransform(A, C, B);
}

// Hermitian short form of the rotated link (5 entries), formed in the
// arithmetic type CT from links and g stored in R
template <typename R>
struct HShort {
  R h0, h3;
  cx<R> h1, h2, h4;
};
// rotated link g(a) U g(b)^dag in the arithmetic type CT
template <typename R, typename CT>
__device__ __forceinline__ void rotated_ct(const CCtx<R> &c, int mu, int s_link,
                                           int sa, int sb, cx<CT> *C) {
  auto up = [](cx<R> a) { return mk<CT>((CT)a.x, (CT)a.y); };
  cx<CT> A[9], B[9];
  {
    cx<R> t[9];
    load_link(c.U, c.V, mu, s_link, t);
#pragma unroll
    for (int e = 0; e < 9; e++) C[e] = up(t[e]);
    load9(c.g, c.V, sa, t);
#pragma unroll
    for (int e = 0; e < 9; e++) A[e] = up(t[e]);
    load9(c.g, c.V, sb, t);
#pragma unroll
    for (int e = 0; e < 9; e++) B[e] = up(t[e]);
  }
  gtransform(A, C, B);
}

template <typename R, typename CT>
__device__ __forceinline__ HShort<CT> rotated_herm(const CCtx<R> &c, int mu,
                                                   int s_link, int sa, int sb) {
  cx<CT> C[9];
  rotated_ct<R, CT>(c, mu, s_link, sa, sb, C);
  HShort<CT> h;
  herm_short(C, h.h0, h.h1, h.h2, h.h3, h.h4);
  return h;
}

// ---------------------------------------------------------------------
// derivative on the rotated links, packed like the Landau fields
// (steep_deriv_CG, src/Gfix/CFACG.c:91-163)
template <typename R, typename CT, int MU>
__device__ __forceinline__ void cderiv_dir(const CCtx<R> &c, const SliceSite &q,
                                           int off, CT &s0, cx<CT> &s1,
                                           cx<CT> &s2, CT &s3, cx<CT> &s4) {
  const int it = sfwd<MU>(q, c.L), bk = sbck<MU>(q, c.L);
  // g(i) U(i) g(i+mu)^dag and g(i-mu) U(i-mu) g(i)^dag
  const HShort<CT> b = rotated_herm<R, CT>(c, MU, off + q.i, off + q.i, off + it);
  const HShort<CT> a = rotated_herm<R, CT>(c, MU, off + bk, off + bk, off + q.i);
  s0 += a.h0 - b.h0;
  s1 = cadd(s1, csub(a.h1, b.h1));
  s2 = cadd(s2, csub(a.h2, b.h2));
  s3 += a.h3 - b.h3;
  s4 = cadd(s4, csub(a.h4, b.h4));
}

// CT: arithmetic type.  With FP32 storage a slice below theta = hp_below is
// worked in FP64 arithmetic: the rotated links g U g^dag of FP32 products
// carry a per-step rounding noise that stalls the FP32 phase near
// theta ~ 1e-8.  `sel` picks the slices of this variant (ArithSel).
template <typename R, typename CT = R>
__global__ void __launch_bounds__(kCoulThreads, 4) k_cderiv(CCtx<R> c, int sel) {
  const int t = blockIdx.y;
  if (c.sl[t].mode == SL_DONE || arith_skip(sel, c.sl[t].tr, c.cs->hp_below))
    return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // in-slice site
  if (i >= c.Lcu) return;
  const SliceSite q = slice_site(i, c.L);
  const int off = t * c.Lcu;
  CT s0 = 0, s3 = 0;
  cx<CT> s1 = mk<CT>(0, 0), s2 = mk<CT>(0, 0), s4 = mk<CT>(0, 0);
  cderiv_dir<R, CT, 0>(c, q, off, s0, s1, s2, s3, s4);
  cderiv_dir<R, CT, 1>(c, q, off, s0, s1, s2, s3, s4);
  cderiv_dir<R, CT, 2>(c, q, off, s0, s1, s2, s3, s4);
  // pack: in0 = i Re s0 - Re s3, in_k = i Re s_k - Im s_k (CFACG.c:144-150)
  cx<R> *f = pick(c.fb, c.st->parity);
  const size_t V = c.V, s = off + i;
  f[s] = mk<R>((R)-s3, (R)s0);
  f[V + s] = mk<R>((R)-s1.y, (R)s1.x);
  f[2 * V + s] = mk<R>((R)-s2.y, (R)s2.x);
  f[3 * V + s] = mk<R>((R)-s4.y, (R)s4.x);
}

// The sums of the accelerated field, insum (sum_DER2 / sum_PR, one norm) and
// sum_conj (src/Gfix/CFACG.c:165-258), come from the inverse xy FFT pass
// (prsum = 1): its per-plane partials of slice t are the planes
// t Lz .. t Lz + Lz - 1 of each of the 4 fields.

// sn = in + beta sn_old at site s (the same fma form as the Landau kernels);
// an SD step takes sn = in without reading sn_old
template <typename R>
__device__ __forceinline__ void cdir(const cx<R> *in, const cx<R> *so, R beta,
                                     bool sd, size_t s, size_t V, cx<R> *f) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const cx<R> a = in[k * V + s];
    if (sd) {
      f[k] = a;
    } else {
      const cx<R> b = so[k * V + s];
      f[k] = mk<R>(fma(beta, b.x, a.x), fma(beta, b.y, a.y));
    }
  }
}

// direction sn = in + beta_t sn_old (an SD step takes sn = in), written for
// every live slice, and the line-search probes of line_search_Coulomb
// (src/Gfix/line_search.c:141-271) at 0.17 and 0.34 as differences to the
// alpha = 0 value; each link counted once (the forward links of every site,
// the same set the reference's draughtboard visits).  Per link the rotated
// link C = g(x) U g(x+mu)^dag is formed once and serves both probes; the
// probe gauge matrices of the site itself wait in shared memory.
// CT: arithmetic type of the probes (FP64 for FP32 storage below hp_below,
// as in k_cderiv); `sel` picks the slices of this variant.
template <typename R, typename CT = R>
__global__ void __launch_bounds__(kCoulThreads, 3) k_cprobe(CCtx<R> c, int sel) {
  __shared__ cx<CT> sA[2][9][kCoulThreads];
  const int t = blockIdx.y;
  if (arith_skip(sel, c.sl[t].tr, c.cs->hp_below)) return;
  double v[2] = {0.0, 0.0};
  const Slice &S = c.sl[t];
  const bool live = S.mode != SL_DONE;
  const bool probes = live && S.use_ls;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (live && i < c.Lcu) {
    const int par = c.st->parity, spar = c.st->sparity;
    const cx<R> *in = pick(c.fb, par), *so = pick(c.sb, spar);
    cx<R> *sn = pick(c.sb, spar ^ 1);
    const R beta = (R)S.beta;
    const bool sdstep = S.sd != 0;
    const int off = t * c.Lcu;
    cx<R> f[4];
    cdir(in, so, beta, sdstep, (size_t)off + i, (size_t)c.V, f);
#pragma unroll
    for (int k = 0; k < 4; k++) sn[(size_t)k * c.V + off + i] = f[k];
    if (probes) {
      auto up = [](cx<R> a) { return mk<CT>((CT)a.x, (CT)a.y); };
      const CT al0 = CT(0.17), al1 = CT(0.34);
#pragma unroll 1
      for (int k = 0; k < 2; k++) {
        cx<CT> A[9];
        set_gauge(A, up(f[0]), up(f[1]), up(f[2]), up(f[3]), k ? al1 : al0);
#pragma unroll
        for (int e = 0; e < 9; e++) sA[k][e][threadIdx.x] = A[e];
      }
      const SliceSite q = slice_site(i, c.L);
      CT d[2] = {0, 0};
#pragma unroll 1
      for (int mu = 0; mu < 3; mu++) {
        const int it = sfwd_rt(q, c.L, mu);
        cx<CT> Cd[9];
        rotated_ct<R, CT>(c, mu, off + i, off + i, off + it, Cd);
        const CT t0 = Cd[0].x + Cd[4].x + Cd[8].x;
        cx<R> fy[4];
        cdir(in, so, beta, sdstep, (size_t)off + it, (size_t)c.V, fy);
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
          cx<CT> A[9], Bm[9];
#pragma unroll
          for (int e = 0; e < 9; e++) A[e] = sA[k][e][threadIdx.x];
          set_gauge(Bm, up(fy[0]), up(fy[1]), up(fy[2]), up(fy[3]), k ? al1 : al0);
          d[k] += re_tr_abc_dag(A, Cd, Bm) - t0;
        }
      }
      v[0] = d[0];
      v[1] = d[1];
    }
  }
  if (probes) block_sum_store<2>(v, c.part + 2 * ((size_t)t * c.nbs + blockIdx.x));
}

// g(x) <- reunit(1 + alpha_t sn(x)) g(x) (exponentiate_gauge_CG,
// src/Gfix/line_search.c:101-115)
template <typename R>
__global__ void __launch_bounds__(kCoulThreads) k_cupdate(CCtx<R> c) {
  const int t = blockIdx.y;
  const Slice &S = c.sl[t];
  if (S.mode == SL_DONE) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.Lcu) return;
  const size_t V = c.V, s = (size_t)t * c.Lcu + i;
  const cx<R> *d = pick(c.sb, c.st->sparity ^ 1);
  cx<R> A[9], G[9], r[9];
  set_gauge(A, d[s], d[V + s], d[2 * V + s], d[3 * V + s], (R)S.alpha);
  load9(c.g, c.V, (int)s, G);
  multab(r, A, G);
  // FP32: the product of many rounded SU(3) factors drifts off the group
  // (~1e-7 a step) and the derivative assumes a unitary g; FP64 keeps GLU's
  // plain product
  if constexpr (sizeof(R) == 4) gram_reunit(r);
  store9(c.g, c.V, (int)s, r);
}

// per-slice housekeeping at the end of a run: reunitarise g_t and check its
// norm (adequate_solution, src/Gfix/CFACG.c:432-456), or replace g_t by
// random SU(3) matrices for a restart (steep_fix, CFACG.c:507-522; our own
// generator, not GLU's RNG stream)
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename R>
__global__ void __launch_bounds__(kCoulThreads) k_cmaint(CCtx<R> c, int what) {
  const int t = blockIdx.y;
  Slice &S = c.sl[t];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.Lcu || S.mode == SL_DONE) return;
  const int s = t * c.Lcu + i;
  if (what == 0 && S.reunit) {
    cx<R> G[9];
    load9(c.g, c.V, s, G);
    gram_reunit(G);
    store9(c.g, c.V, s, G);
    double sum = 0.0;
#pragma unroll
    for (int e = 0; e < 9; e++) sum += (double)G[e].x * G[e].x + (double)G[e].y * G[e].y;
    const double lim = (double)(S.iter > 0 ? S.iter : 1) * c.cs->prec_tol;
    if (fabs(sum - 3.0) > lim) atomicOr(&S.bad, 1);
  } else if (what == 1 && S.randomize) {
    cx<R> G[9];
    unsigned long long h = mix64(c.cs->seed ^ mix64(((unsigned long long)t << 40) ^
                                                    ((unsigned long long)S.control << 32) ^
                                                    (unsigned long long)i));
#pragma unroll
    for (int e = 0; e < 9; e++) {
      h = mix64(h);
      const double u1 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      h = mix64(h);
      const double u2 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      const double rad = sqrt(-2.0 * log(u1));
      G[e] = mk<R>((R)(rad * cospi(2.0 * u2)), (R)(rad * sinpi(2.0 * u2)));
    }
    gram_reunit(G);
    store9(c.g, c.V, s, G);
  }
}

enum CoulOp : int { C_SUMS = 0, C_PROBES = 1, C_END1 = 2, C_END2 = 3 };

// one warp per slice: fixed-order sums of the slice's partials (each lane
// a strided subset in order, then a fixed shuffle tree), and GLU's control
// flow of steep_step_FACG / _FASD and steep_fix (src/Gfix/CFACG.c:285-529)
// on lane 0.
// Partials: C_SUMS reads the inverse xy FFT pass's per-plane pairs (plane
// index field * nplanes + t * lz + z), C_PROBES the probe kernel's per-block
// pairs (t * nbs + block).
constexpr int kCScalarSlices = 4;  // slices (warps) per block

__global__ void __launch_bounds__(32 * kCScalarSlices)
    k_cscalar(CoulState *cs, Slice *sl, const double *part, int nbs, int lz,
              int nplanes, int op, double Lcu, DevState *st) {
  const int t = blockIdx.x * kCScalarSlices + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t < cs->nslices) {
    Slice &S = sl[t];
    if (S.mode != SL_DONE) {
      double a0 = 0.0, a1 = 0.0;
      if (op == C_SUMS) {
        const int n = 4 * lz;  // (field, z) pairs, field-major
        for (int j = lane; j < n; j += 32) {
          const int f = j / lz, z = j % lz;
          const size_t b = (size_t)f * nplanes + (size_t)t * lz + z;
          a0 += part[2 * b];
          a1 += part[2 * b + 1];
        }
      } else if (op == C_PROBES) {
        constexpr int kU = 4;
        for (int b0 = lane; b0 < nbs; b0 += 32 * kU) {
          double x0[kU], x1[kU];
#pragma unroll
          for (int k = 0; k < kU; k++) {
            const int b = b0 + 32 * k;
            x0[k] = b < nbs ? part[2 * ((size_t)t * nbs + b)] : 0.0;
            x1[k] = b < nbs ? part[2 * ((size_t)t * nbs + b) + 1] : 0.0;
          }
#pragma unroll
          for (int k = 0; k < kU; k++) {
            a0 += x0[k];
            a1 += x1[k];
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, o);
        a1 += __shfl_down_sync(0xffffffffu, a1, o);
      }
      if (lane != 0) return;
      switch (op) {
        case C_SUMS: {
          S.insum = a0;
          S.sumconj = a1;
          S.tr = a0 / (3.0 * Lcu);  // GFNORM_COULOMB
          if (S.sd) {
            S.inold = a0;
            S.beta = 0.0;
            // FACG's SD start always searches (CFACG.c:318); FASD steps
            // search unless GLU_GFIX_SD (CFACG.c:270-280)
            S.use_ls = cs->facg ? 1 : !cs->sd_fixed;
          } else {
            const double b = S.sumconj / S.inold;
            double beta = (b < 0.0) ? 0.0 : b;
            if (S.tr < cs->cg_tol) beta = S.insum / S.inold;
            S.beta = beta;
            S.inold = S.insum;
            S.use_ls = S.tr > cs->cg_tol;
          }
          if (cs->traj && S.traj_len < cs->traj_cap)
            cs->traj[(size_t)t * cs->traj_cap + S.traj_len++] = S.tr;
          break;
        }
        case C_PROBES: {
          if (S.use_ls) {
            const double al[3] = {0.0, 0.17, 0.34};
            const double f[3] = {0.0, -a0, -a1};
            S.alpha = approx_minimum(al, f);
          } else {
            S.alpha = cs->gf_alpha;
          }
          break;
        }
        case C_END1: {
          S.reunit = 0;
          S.bad = 0;
          S.randomize = 0;
          if (cs->facg && S.sd) {
            S.sd = 0;  // the SD start is not counted
            break;
          }
          S.iter++;
          if (cs->stall_window > 0 && S.tr > cs->acc) {
            if (S.tr < 0.9 * S.best_tr) {
              S.best_tr = S.tr;
              S.since_best = 0;
            } else {
              S.since_best++;
            }
            if (S.best_tr < cs->stall_floor &&
                (S.since_best >= cs->stall_window || S.tr > cs->blowup * S.best_tr)) {
              S.sd = -1;  // ends the run, no restart: the FP64 phase goes on
              break;
            }
          }
          if ((S.tr > cs->acc) && (S.iter < cs->max_iters)) break;
          S.reunit = S.tr < cs->acc;  // run ended: adequate_solution first
          S.sd = -1;                  // marks "ended" for C_END2
          break;
        }
        case C_END2: {
          if (S.sd != -1) break;
          const long long loc = S.iter;
          const bool fin = isfinite(S.tr);
          if (S.bad) S.trans = 1;
          S.sd = 1;
          S.iter = 0;
          if (loc >= cs->max_iters) {
            if (S.tr < 1E4 * cs->acc && fin) {  // continuation run
              S.tot += loc;
              break;
            }
            if (S.tr > cs->acc || !fin) S.trans = 1;
          }
          if (S.control < 8 && S.trans) {  // random restart
            S.randomize = 1;
            S.trans = 0;
            S.tot += loc;
            S.control++;
            break;
          }
          S.tot += loc;
          S.iter = loc;
          S.mode = SL_DONE;
          cs->done_mask[t] = 1;
          // the slice that ends last stops the whole sequence
          if (atomicSub(&cs->active, 1) == 1) st->done = 1;
          break;
        }
      }
    }
  }
}

// the slice transforms of Coulomb_FA (gtransform_slice, src/Gfix/gtrans.c:
// 214-238): U_i(x,t) <- g_t(x) U_i(x,t) g_t(x+i)^dag for i < 3 and
// U_t(x,t) <- g_t(x) U_t(x,t) g_{t+1}(x)^dag.  ALL_T: every temporal link,
// periodic in t (a whole lattice); otherwise the last slice's temporal links
// are left for k_cfinish_aos (a block of slices whose successor slice lives
// elsewhere).
template <typename R, int MU>
__device__ __forceinline__ void cslice_link(const CCtx<R> &c, const SliceSite &q,
                                            int s, int t, const cx<R> *A) {
  const int nb = MU < 3 ? t * c.Lcu + sfwd<(MU < 3 ? MU : 0)>(q, c.L)
                        : ((t + 1) % c.L[3]) * c.Lcu + q.i;
  cx<R> B[9], U[9];
  load9(c.g, c.V, nb, B);
  load_link(c.U, c.V, MU, s, U);
  gtransform(A, U, B);
  store_link(c.U, c.V, MU, s, U);
}

template <typename R>
__global__ void __launch_bounds__(kCoulThreads) k_cslice_transform(CCtx<R> c,
                                                                   int all_t) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.V) return;
  const int t = s / c.Lcu;
  const SliceSite q = slice_site(s - t * c.Lcu, c.L);
  cx<R> A[9];
  load9(c.g, c.V, s, A);
  cslice_link<R, 0>(c, q, s, t, A);
  cslice_link<R, 1>(c, q, s, t, A);
  cslice_link<R, 2>(c, q, s, t, A);
  if (all_t || t < c.L[3] - 1) cslice_link<R, 3>(c, q, s, t, A);
}

// the temporal links of the last local slice, U_t <- g_last U_t g_next^dag,
// in the caller's AoS links (double[V][4][9][2]); g_last and g_next are the
// fields of that slice and of the following one (double[9][Lcu][2])
__global__ void __launch_bounds__(kCoulThreads)
    k_cfinish_aos(double2 *links, const double2 *g_last, const double2 *g_next,
                  int V, int Lcu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Lcu) return;
  const int s = V - Lcu + i;
  cx<double> A[9], B[9], U[9];
#pragma unroll
  for (int e = 0; e < 9; e++) {
    const double2 a = g_last[(size_t)e * Lcu + i];
    const double2 b = g_next[(size_t)e * Lcu + i];
    A[e] = mk<double>(a.x, a.y);
    B[e] = mk<double>(b.x, b.y);
  }
  double2 *u = links + ((size_t)s * 4 + 3) * 9;
#pragma unroll
  for (int e = 0; e < 9; e++) U[e] = mk<double>(u[e].x, u[e].y);
  gtransform(A, U, B);
#pragma unroll
  for (int e = 0; e < 9; e++) u[e] = make_double2(U[e].x, U[e].y);
}

// g of local slice t, exported as double[9][Lcu][2]
__global__ void k_cexport_slice(const cx<double> *g, double2 *out, int V,
                                int Lcu, int t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Lcu) return;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    const cx<double> v = g[(size_t)e * V + (size_t)t * Lcu + i];
    out[(size_t)e * Lcu + i] = make_double2(v.x, v.y);
  }
}

// in / in_old and sn ping-pong after every step of every live slice
__global__ void k_cflip(DevState *st) {
  if (st->done) return;
  st->parity ^= 1;
  st->sparity ^= 1;
}

template <typename R>
__global__ void k_cinit(CCtx<R> c) {
  const size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (s >= (size_t)c.V) return;
  cx<R> G[9];
  set_identity(G);
  store9(c.g, c.V, (int)s, G);
}

}  // namespace gfix
