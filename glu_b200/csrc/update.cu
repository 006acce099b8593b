// Quenched SU(3) configuration generation on the GPU: GLU's heatbath +
// over-relaxation update (hb_update, src/Update/KPHB.c:123-257), the step
// before gauge fixing.
//
//   heatbath        hb_lattice (src/Update/hb.c:146-194): per link the
//                   Wilson staple (all_staples, src/Smear/staples.c:32-79),
//                   then for each of the three SU(2) subgroups the
//                   normalised subgroup of U staple^dag (only_subgroup,
//                   src/Update/SU2_rotate_SSE.c:75-216), a Kennedy-Pendleton
//                   draw (KP / generate_SU2, hb.c:40-127, at most 43 draws)
//                   and the rotation (su2_rotate, SU2_rotate_SSE.c:287-390);
//                   the link is reunitarised afterwards (gram_reunit)
//   over-relaxation OR_lattice (src/Update/relax.c:83-114): the same with
//                   the microcanonical reflection (relax.c:32-43) in place
//                   of the draw, no reunitarisation
//
// Order: GLU updates every link of direction mu of one draughtboard colour,
// then the next colour, then the next direction (hb.c:176-190); links of
// one colour and direction share no staple, so each (mu, colour) step is
// one launch with one thread per link.  Colours are the site parity for
// even extents (draughtboard.c:51-73); odd extents are rejected.
//
// Layout in HBM: links checkerboard-ordered SoA, U[mu][element][parity]
// [V/2] complex FP64 -- the threads of a launch read their own links and
// those of their neighbours with unit stride.  GLU's AoS links convert in
// and out at the boundary.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011), counter-based: the key is
// the seed, the counter (link, iteration, draw), so a run is reproducible
// and any iteration can be restarted from (seed, iteration) alone.  GLU's
// own per-thread generator stream is not reproduced: the heatbath agrees
// with GLU in distribution (plaquette), the over-relaxation value for value.

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/glu_gfix.h"
#include "su3.cuh"

namespace gfix {
void count_launches(unsigned long long n);  // gfix.cu
namespace upd {

thread_local std::string t_err;

int ufail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
  return -1;
}

#define UCK(call)                                                       \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess)                                              \
      return ufail("%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                   cudaGetErrorString(e_));                             \
  } while (0)

using C2 = cx<double>;

constexpr double kTwoPi = 6.283185307179586;  // GLU's TWOPI
// NHBMAX = 42 (hb.c:33) bounds the loop counter of hb.c:86-90, which
// evaluates one more draw before the bound stops it: 43 draws at most
constexpr int kMaxTries = 43;
constexpr int kThreads = 128;
#ifndef UPD_MINB
#define UPD_MINB 3  // resident blocks asked of the register allocator
#endif

// ---------------------------------------------------------------------
// Philox4x32-10

struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t *hi,
                                                 uint32_t *lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {  // constant trip count: unrolled by nvcc
    uint32_t h0, l0, h1, l1;
    mulhilo(M0, c.x, &h0, &l0);
    mulhilo(M1, c.z, &h1, &l1);
    c = U4{h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform doubles in (0, 1) (53 random bits, never 0 or 1), two per block
struct Rng {
  U4 ctr;
  uint32_t k0, k1;
  double second = 0.0;
  bool have = false;  // `second` holds an unused number
  __device__ __forceinline__ double next() {
    if (have) {
      have = false;
      return second;
    }
    const U4 r = philox4x32_10(ctr, k0, k1);
    ctr.w++;
    const uint64_t a = ((uint64_t)r.x << 32 | r.y) >> 11;
    const uint64_t b = ((uint64_t)r.z << 32 | r.w) >> 11;
    second = ((double)b + 0.5) * 0x1.0p-53;
    have = true;
    return ((double)a + 0.5) * 0x1.0p-53;
  }
};

// ---------------------------------------------------------------------
// geometry of the checkerboard layout

struct UpdCtx {
  int L[4];
  int V, Vh;      // sites, sites per parity
  C2 *U;          // [4][9][2][Vh]
  double *part;   // per-block partial sums
};

// site coordinates of index h of parity p (Lx even: sites 2k and 2k+1
// along x have opposite parities, so h = site / 2 within each parity)
__device__ __forceinline__ void cb_coords(const UpdCtx &c, int p, int h, int x[4]) {
  const int hx = c.L[0] >> 1;
  int r = h / hx;
  const int x2 = h - r * hx;
  x[1] = r % c.L[1];
  r /= c.L[1];
  x[2] = r % c.L[2];
  x[3] = r / c.L[2];
  const int b = (p + x[1] + x[2] + x[3]) & 1;
  x[0] = 2 * x2 + b;
}

// (parity, half index) of the site at x
__device__ __forceinline__ int cb_index(const UpdCtx &c, const int x[4], int *p) {
  *p = (x[0] + x[1] + x[2] + x[3]) & 1;
  return (x[0] >> 1) + (c.L[0] >> 1) * (x[1] + c.L[1] * (x[2] + c.L[2] * x[3]));
}

__device__ __forceinline__ void load_cb(const UpdCtx &c, int mu, int p, int h, C2 *u) {
  const C2 *q = c.U + ((size_t)mu * 9 * 2 + p) * c.Vh + h;
#pragma unroll
  for (int e = 0; e < 9; e++) u[e] = q[(size_t)e * 2 * c.Vh];
}

__device__ __forceinline__ void store_cb(const UpdCtx &c, int mu, int p, int h, const C2 *u) {
  C2 *q = c.U + ((size_t)mu * 9 * 2 + p) * c.Vh + h;
#pragma unroll
  for (int e = 0; e < 9; e++) q[(size_t)e * 2 * c.Vh] = u[e];
}

// the link U_mu at x shifted by +-1 along nu (and optionally along mu)
__device__ __forceinline__ void load_at(const UpdCtx &c, int mu, const int x[4], C2 *u) {
  int p;
  const int h = cb_index(c, x, &p);
  load_cb(c, mu, p, h, u);
}

// ---------------------------------------------------------------------
// SU(3) and SU(2) pieces

__device__ __forceinline__ C2 cmul2(C2 a, C2 b) {
  return mk<double>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b), conj(a) * b
__device__ __forceinline__ C2 cmulc2(C2 a, C2 b) {
  return mk<double>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ C2 ccmul2(C2 a, C2 b) {
  return mk<double>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ C2 add2(C2 a, C2 b) { return mk<double>(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ C2 sub2(C2 a, C2 b) { return mk<double>(a.x - b.x, a.y - b.y); }

// o = a b
__device__ __forceinline__ void m_ab(C2 *o, const C2 *a, const C2 *b) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int s = 0; s < 3; s++)
      o[3 * r + s] = add2(add2(cmul2(a[3 * r], b[s]), cmul2(a[3 * r + 1], b[3 + s])),
                          cmul2(a[3 * r + 2], b[6 + s]));
}
// o += a b^dag
__device__ __forceinline__ void m_abdag_acc(C2 *o, const C2 *a, const C2 *b) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int s = 0; s < 3; s++)
      o[3 * r + s] = add2(o[3 * r + s],
                          add2(add2(cmulc2(a[3 * r], b[3 * s]), cmulc2(a[3 * r + 1], b[3 * s + 1])),
                               cmulc2(a[3 * r + 2], b[3 * s + 2])));
}
// o = a^dag b
__device__ __forceinline__ void m_adagb(C2 *o, const C2 *a, const C2 *b) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int s = 0; s < 3; s++)
      o[3 * r + s] = add2(add2(ccmul2(a[r], b[s]), ccmul2(a[3 + r], b[3 + s])),
                          ccmul2(a[6 + r], b[6 + s]));
}
// o += a b
__device__ __forceinline__ void m_ab_acc(C2 *o, const C2 *a, const C2 *b) {
  C2 t[9];
  m_ab(t, a, b);
#pragma unroll
  for (int e = 0; e < 9; e++) o[e] = add2(o[e], t[e]);
}

__device__ __forceinline__ int fwd(int v, int L) { return v + 1 == L ? 0 : v + 1; }
__device__ __forceinline__ int bck(int v, int L) { return v == 0 ? L - 1 : v - 1; }

// the Wilson staple of U_MU(x): sum over nu != MU of
// U_nu(x) U_MU(x+nu) U_nu(x+MU)^dag + U_nu(x-nu)^dag U_MU(x-nu) U_nu(x-nu+MU)
// (MU a template constant and the nu loop unrolled: every coordinate index
// is a compile-time constant, nothing goes to local memory)
template <int MU>
__device__ __forceinline__ void staple(const UpdCtx &c, const int x[4], C2 *st) {
#pragma unroll
  for (int e = 0; e < 9; e++) st[e] = mk<double>(0., 0.);
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    if (nu == MU) continue;
    C2 a[9], b[9], t[9];
    int y[4] = {x[0], x[1], x[2], x[3]};
    // top
    load_at(c, nu, y, a);
    y[nu] = fwd(x[nu], c.L[nu]);
    load_at(c, MU, y, b);
    m_ab(t, a, b);
    y[nu] = x[nu];
    y[MU] = fwd(x[MU], c.L[MU]);
    load_at(c, nu, y, a);
    m_abdag_acc(st, t, a);
    // bottom
    y[MU] = x[MU];
    y[nu] = bck(x[nu], c.L[nu]);
    load_at(c, nu, y, a);
    load_at(c, MU, y, b);
    m_adagb(t, a, b);
    y[MU] = fwd(x[MU], c.L[MU]);
    load_at(c, nu, y, a);
    m_ab_acc(st, t, a);
  }
}

// rows (r0, r1) of an SU(2) subgroup: 0 -> (0, 1), 1 -> (1, 2), 2 -> (2, 0)
// as only_subgroup / su2_rotate lay them out
__device__ __forceinline__ void subgroup(const C2 *U, const C2 *S, int g, C2 *s0, C2 *s1,
                                         double *scale) {
  C2 m0 = mk<double>(0., 0.), m1 = mk<double>(0., 0.);
  if (g < 2) {
    const int a = 3 * g, b = 3 * g + 3;  // rows g, g+1
    C2 t0 = mk<double>(0., 0.), t3 = t0, t1 = t0, t2 = t0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      t0 = add2(t0, cmulc2(U[a + k], S[a + k]));  // U[g][k] conj S[g][k]
      t3 = add2(t3, ccmul2(U[b + k], S[b + k]));  // conj U[g+1][k] S[g+1][k]
      t1 = add2(t1, cmulc2(U[a + k], S[b + k]));
      t2 = add2(t2, ccmul2(U[b + k], S[a + k]));
    }
    m0 = add2(t0, t3);
    m1 = sub2(t1, t2);
  } else {
    // rows 0 and 2 with the roles of the two rows exchanged (rotation 3)
    C2 t0 = mk<double>(0., 0.), t3 = t0, t1 = t0, t2 = t0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      t3 = add2(t3, ccmul2(U[k], S[k]));          // conj U[0][k] S[0][k]
      t0 = add2(t0, cmulc2(U[6 + k], S[6 + k]));  // U[2][k] conj S[2][k]
      t1 = add2(t1, cmulc2(U[6 + k], S[k]));
      t2 = add2(t2, ccmul2(U[k], S[6 + k]));
    }
    m0 = add2(t3, t0);
    m1 = sub2(t1, t2);
  }
  const double z = 1.0 / sqrt(m0.x * m0.x + m1.x * m1.x + (m0.y * m0.y + m1.y * m1.y));
  *s0 = mk<double>(m0.x * z, m0.y * z);
  *s1 = mk<double>(m1.x * z, m1.y * z);
  *scale = z;
}

// U <- R U with R the SU(2) element (s0, s1) in subgroup g
__device__ __forceinline__ void rotate(C2 *U, int g, C2 s0, C2 s1) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    if (g < 2) {
      const C2 a = U[3 * g + j], b = U[3 * g + 3 + j];
      U[3 * g + j] = add2(cmul2(s0, a), cmul2(s1, b));
      U[3 * g + 3 + j] = sub2(ccmul2(s0, b), ccmul2(s1, a));
    } else {
      const C2 a = U[j], b = U[6 + j];
      U[j] = sub2(ccmul2(s0, a), ccmul2(s1, b));
      U[6 + j] = add2(cmul2(s0, b), cmul2(s1, a));
    }
  }
}

// Kennedy-Pendleton draw of d = 1 - a0 (hb.c:40-49, 83-97): up to 43 draws,
// the last one kept if none is accepted
__device__ __forceinline__ double kp_draw(Rng &g, double norm) {
  double d = 0.0;
  for (int it = 0; it < kMaxTries; it++) {
    const double x4 = g.next();
    const double x3 = cos(kTwoPi * g.next());
    const double l1 = log(g.next()), l2 = log(g.next());
    d = -(l1 + l2 * x3 * x3) * norm;
    if (!((1. - 0.5 * d) < x4 * x4)) break;
  }
  return d;
}

// heatbath SU(2) element times the conjugate of the normalised staple
// subgroup (generate_SU2, hb.c:99-127)
__device__ __forceinline__ void hb_su2(Rng &g, double norm, C2 *s0, C2 *s1) {
  const double d = kp_draw(g, norm);
  const double a0 = 1.0 - d;
  const double ar2 = fabs(1.0 - a0 * a0);
  const double a3 = sqrt(ar2) * (2.0 * g.next() - 1.0);
  const double rho = sqrt(fabs(ar2 - a3 * a3));
  const double xr2 = kTwoPi * g.next();
  double a1, a2;
  sincos(xr2, &a2, &a1);
  a1 *= rho;
  a2 *= rho;
  const double rS0 = s0->x, iS0 = s0->y, rS1 = s1->x, iS1 = s1->y;
  *s0 = mk<double>(a0 * rS0 + a3 * iS0 + a2 * rS1 + a1 * iS1,
                   -a0 * iS0 + rS0 * a3 - a2 * iS1 + rS1 * a1);
  *s1 = mk<double>(-a0 * rS1 + a3 * iS1 + a2 * rS0 - a1 * iS0,
                   -a0 * iS1 - a3 * rS1 + a2 * iS0 + a1 * rS0);
}

// microcanonical reflection (relax.c:32-43)
__device__ __forceinline__ void or_su2(C2 *s0, C2 *s1) {
  const double z = s0->x * s0->x - s0->y * s0->y - s1->x * s1->x - s1->y * s1->y;
  const double r = s0->x;
  *s1 = mk<double>(-2. * r * s1->x, -2. * r * s1->y);
  *s0 = mk<double>(z, -(2. * r * s0->y));
}

// ---------------------------------------------------------------------
// kernels

// one (direction, parity) step of a heatbath (HB) or over-relaxation sweep
// over the links U_mu of parity p; counter (link, mu and parity, iteration,
// draw) for the generator
template <bool HB, int MU>
__global__ void __launch_bounds__(kThreads, UPD_MINB) k_update(UpdCtx c, int p, double invbeta,
                                                    uint32_t k0, uint32_t k1, uint32_t iter) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= c.Vh) return;
  int x[4];
  cb_coords(c, p, h, x);
  C2 st[9], U[9];
  staple<MU>(c, x, st);
  load_cb(c, MU, p, h, U);
  Rng g;
  g.ctr = U4{(uint32_t)h, (uint32_t)(2 * MU + p), iter, 0u};
  g.k0 = k0;
  g.k1 = k1;
#pragma unroll
  for (int sg = 0; sg < 3; sg++) {
    C2 s0, s1;
    double scale;
    subgroup(U, st, sg, &s0, &s1, &scale);
    if (HB)
      hb_su2(g, invbeta * scale, &s0, &s1);
    else
      or_su2(&s0, &s1);
    rotate(U, sg, s0, s1);
  }
  if (HB) gram_reunit(U);
  store_cb(c, MU, p, h, U);
}

// per-block partial sums of Re tr of the six plaquettes at every site
// (av_plaquette, src/Field/plaqs_links.c:243-265)
__global__ void __launch_bounds__(kThreads) k_plaq(UpdCtx c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < c.V) {
    const int p = t / c.Vh, h = t - p * c.Vh;
    int x[4];
    cb_coords(c, p, h, x);
#pragma unroll 1
    for (int mu = 1; mu < 4; mu++)
#pragma unroll 1
      for (int nu = 0; nu < mu; nu++) {
        C2 a[9], b[9], t1[9], t2[9];
        int y[4] = {x[0], x[1], x[2], x[3]};
        load_cb(c, mu, p, h, a);
        y[mu] = (x[mu] + 1) % c.L[mu];
        load_at(c, nu, y, b);
        m_ab(t1, a, b);  // U_mu(x) U_nu(x+mu)
        y[mu] = x[mu];
        y[nu] = (x[nu] + 1) % c.L[nu];
        load_at(c, mu, y, a);
        load_cb(c, nu, p, h, b);
        m_ab(t2, b, a);  // U_nu(x) U_mu(x+nu)
        // Re tr(t1 t2^dag)
#pragma unroll
        for (int e = 0; e < 9; e++) v += t1[e].x * t2[e].x + t1[e].y * t2[e].y;
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __shared__ double sw[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; w++) s += sw[w];
    c.part[blockIdx.x] = s;
  }
}

// GLU's AoS links <-> the checkerboard layout
__global__ void __launch_bounds__(kThreads) k_to_cb(UpdCtx c, const C2 *aos) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.V) return;
  const int p = t / c.Vh, h = t - p * c.Vh;
  int x[4];
  cb_coords(c, p, h, x);
  const size_t s = x[0] + (size_t)c.L[0] * (x[1] + (size_t)c.L[1] * (x[2] + (size_t)c.L[2] * x[3]));
#pragma unroll 1
  for (int mu = 0; mu < 4; mu++) {
    C2 u[9];
#pragma unroll
    for (int e = 0; e < 9; e++) u[e] = aos[(s * 4 + mu) * 9 + e];
    store_cb(c, mu, p, h, u);
  }
}

__global__ void __launch_bounds__(kThreads) k_from_cb(UpdCtx c, C2 *aos) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.V) return;
  const int p = t / c.Vh, h = t - p * c.Vh;
  int x[4];
  cb_coords(c, p, h, x);
  const size_t s = x[0] + (size_t)c.L[0] * (x[1] + (size_t)c.L[1] * (x[2] + (size_t)c.L[2] * x[3]));
#pragma unroll 1
  for (int mu = 0; mu < 4; mu++) {
    C2 u[9];
    load_cb(c, mu, p, h, u);
#pragma unroll
    for (int e = 0; e < 9; e++) aos[(s * 4 + mu) * 9 + e] = u[e];
  }
}

// ---------------------------------------------------------------------
// host side: one workspace per lattice shape

struct Work {
  UpdCtx c{};
  cudaStream_t s = nullptr;
  C2 *d_aos = nullptr;
  int nb_half = 0, nb_all = 0;
  std::vector<double> part;

  ~Work() {
    cudaFree(c.U);
    cudaFree(c.part);
    cudaFree(d_aos);
    if (s) cudaStreamDestroy(s);
  }

  int init(const size_t *d) {
    size_t V = 1;
    for (int i = 0; i < 4; i++) {
      if (d[i] < 2 || d[i] % 2)
        return ufail("extent %zu of dimension %d: the update needs even extents "
                     "(two draughtboard colours)", d[i], i);
      c.L[i] = (int)d[i];
      V *= d[i];
    }
    if (V > (size_t)INT32_MAX / 4) return ufail("lattice volume %zu too large", V);
    c.V = (int)V;
    c.Vh = c.V / 2;
    nb_half = (c.Vh + kThreads - 1) / kThreads;
    nb_all = (c.V + kThreads - 1) / kThreads;
    UCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    UCK(cudaMalloc(&c.U, V * 36 * sizeof(C2)));
    UCK(cudaMalloc(&c.part, nb_all * sizeof(double)));
    part.resize(nb_all);
    return 0;
  }

  int ensure_aos() {
    if (!d_aos) UCK(cudaMalloc(&d_aos, (size_t)c.V * 36 * sizeof(C2)));
    return 0;
  }

  void to_cb(const C2 *aos) {
    k_to_cb<<<nb_all, kThreads, 0, s>>>(c, aos);
    count_launches(1);
  }
  void from_cb(C2 *aos) {
    k_from_cb<<<nb_all, kThreads, 0, s>>>(c, aos);
    count_launches(1);
  }

  // one sweep in GLU's order: every direction, both colours
  void sweep(bool hb, double invbeta, uint64_t seed, uint32_t iter) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int mu = 0; mu < 4; mu++)
      for (int p = 0; p < 2; p++) {
        auto f = hb ? (mu == 0 ? k_update<true, 0> : mu == 1 ? k_update<true, 1>
                       : mu == 2 ? k_update<true, 2> : k_update<true, 3>)
                    : (mu == 0 ? k_update<false, 0> : mu == 1 ? k_update<false, 1>
                       : mu == 2 ? k_update<false, 2> : k_update<false, 3>);
        f<<<nb_half, kThreads, 0, s>>>(c, p, invbeta, k0, k1, iter);
      }
    count_launches(8);
  }

  // average plaquette, fixed-order sum of the block partials
  int plaquette(double *out) {
    k_plaq<<<nb_all, kThreads, 0, s>>>(c);
    count_launches(1);
    UCK(cudaMemcpyAsync(part.data(), c.part, nb_all * sizeof(double),
                        cudaMemcpyDeviceToHost, s));
    UCK(cudaStreamSynchronize(s));
    double sum = 0.0;
    for (int b = 0; b < nb_all; b++) sum += part[b];
    *out = sum / (3.0 * 6.0 * c.V);
    return 0;
  }

  // iterations of one heatbath sweep and n_or over-relaxation sweeps
  // (update_lattice, KPHB.c:83-99); plaq (may be NULL) after each one
  int run(double beta, size_t iterations, size_t n_or, uint64_t seed, uint64_t first,
          double *plaq) {
    if (!(beta > 0.0)) return ufail("beta %g must be positive", beta);
    const double invbeta = 3.0 / beta;  // NC / beta (KPHB.c:170)
    for (size_t i = 0; i < iterations; i++) {
      sweep(true, invbeta, seed, (uint32_t)(first + i));
      for (size_t k = 0; k < n_or; k++) sweep(false, 0.0, 0, 0);
      if (plaq && plaquette(&plaq[i])) return -1;
    }
    UCK(cudaGetLastError());
    return 0;
  }
};

// one workspace per (device, lattice shape): a workspace's buffers and
// stream belong to the device that was current when it was made
static std::map<std::array<size_t, 5>, std::unique_ptr<Work>> g_work;
static std::mutex g_work_mu;

static Work *work_for(const size_t *dims) {
  if (!dims) {
    ufail("null dims");
    return nullptr;
  }
  for (int i = 0; i < 4; i++)
    if (dims[i] < 2 || dims[i] % 2) {
      ufail("extent %zu of dimension %d: the update needs even extents "
            "(two draughtboard colours)", dims[i], i);
      return nullptr;
    }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    ufail("no CUDA device");
    return nullptr;
  }
  const std::array<size_t, 5> k{(size_t)dev, dims[0], dims[1], dims[2], dims[3]};
  std::lock_guard<std::mutex> lk(g_work_mu);
  auto it = g_work.find(k);
  if (it != g_work.end()) return it->second.get();
  auto w = std::make_unique<Work>();
  if (w->init(dims)) return nullptr;
  return g_work.emplace(k, std::move(w)).first->second.get();
}

}  // namespace upd
}  // namespace gfix

using namespace gfix::upd;

extern "C" {

const char *gfix_update_error(void) { return t_err.c_str(); }

int gfix_heatbath_device(double *d_links, const size_t dims[4], double beta,
                         size_t iterations, size_t n_or, uint64_t seed,
                         uint64_t first_iteration, double *plaquettes) {
  if (!d_links) return ufail("null links");
  Work *w = work_for(dims);
  if (!w) return -1;
  // the library's stream does not synchronise with the caller's: wait for
  // all work on the device, so a kernel that has just written the links
  // (on any stream) has finished before they are read
  UCK(cudaDeviceSynchronize());
  C2 *aos = reinterpret_cast<C2 *>(d_links);
  w->to_cb(aos);
  if (w->run(beta, iterations, n_or, seed, first_iteration, plaquettes)) return -1;
  w->from_cb(aos);
  UCK(cudaStreamSynchronize(w->s));
  UCK(cudaGetLastError());
  return 0;
}

int gfix_heatbath(double *links, const size_t dims[4], double beta, size_t iterations,
                  size_t n_or, uint64_t seed, uint64_t first_iteration,
                  double *plaquettes) {
  if (!links) return ufail("null links");
  Work *w = work_for(dims);
  if (!w || w->ensure_aos()) return -1;
  const size_t bytes = (size_t)w->c.V * 36 * sizeof(C2);
  UCK(cudaMemcpyAsync(w->d_aos, links, bytes, cudaMemcpyHostToDevice, w->s));
  w->to_cb(w->d_aos);
  if (w->run(beta, iterations, n_or, seed, first_iteration, plaquettes)) return -1;
  w->from_cb(w->d_aos);
  UCK(cudaMemcpyAsync(links, w->d_aos, bytes, cudaMemcpyDeviceToHost, w->s));
  UCK(cudaStreamSynchronize(w->s));
  UCK(cudaGetLastError());
  return 0;
}

int gfix_overrelax(double *links, const size_t dims[4], size_t sweeps) {
  if (!links) return ufail("null links");
  Work *w = work_for(dims);
  if (!w || w->ensure_aos()) return -1;
  const size_t bytes = (size_t)w->c.V * 36 * sizeof(C2);
  UCK(cudaMemcpyAsync(w->d_aos, links, bytes, cudaMemcpyHostToDevice, w->s));
  w->to_cb(w->d_aos);
  for (size_t k = 0; k < sweeps; k++) w->sweep(false, 0.0, 0, 0);
  w->from_cb(w->d_aos);
  UCK(cudaMemcpyAsync(links, w->d_aos, bytes, cudaMemcpyDeviceToHost, w->s));
  UCK(cudaStreamSynchronize(w->s));
  UCK(cudaGetLastError());
  return 0;
}

void gfix_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  const U4 r = philox4x32_10(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

void gfix_update_release(void) {
  std::lock_guard<std::mutex> lk(g_work_mu);
  g_work.clear();
}

}  // extern "C"
