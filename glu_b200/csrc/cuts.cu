// Momentum-space gluon measurements on the GPU: GLU's cuts_struct
// (src/Cuts/cuts.c:110-184) for CUTTYPE = GLUON_PROPS (glueprop.c),
// EXCEPTIONAL (MOMgg.c) and FIELDS (cut_output.c:337-366), in GLU's
// default build (SIN_MOM, backward transform, matrix contraction).
//
// Pipeline (FP64 throughout):
//   k_cut_xy4_ct  Lie field of every link -- FIELD_DEFINITION LINEAR
//                 (Hermitian_proj, exactQ.c:358-385) or LOGARITHMIC
//                 (exact_log_slow, exactQ.c:157-240) -- packed per direction
//                 in 4 complex fields (A00 + i A11, A01, A02, A12: the
//                 traceless Hermitian matrix's 8 reals), then the x and y
//                 transforms of the four fields of one direction of one xy
//                 plane per block.  The links are read once, straight into
//                 the transform.
//   k_cut_xy      the same per field (planes too large for four tiles, and
//                 the generic extents); with the logarithm, k_cut_log_pack
//                 writes the packed fields first
//   k_cut_zt      z and t transforms of tiles of x columns
//                 (both also as k_cut_*_ct with compile-time extents)
//   k_cut_gather  per listed momentum: A_mu(p) for all 9 colour entries
//                 from the packed transforms at p and -p (the transform of
//                 a real field R obeys R(-p) = conj R(p), and of conj(f)
//                 it is conj f(-p)), times e^{i p_mu / 2} (pspace_landau.c)
//                 and the p-space gauge error term
//   k_cut_props   transverse / longitudinal propagators (GLUON_PROPS)
//   k_cut_momgg   MOMgg g2, g3 (EXCEPTIONAL)
//
// GLU transforms each of the 36 colour entries separately (36 complex
// FFTs); the packing needs 16.  Transforms follow GLU's backward FFTW
// plan: sum_x f(x) e^{+ipx}, unnormalised.  The momentum list is host
// code (cut_routines.c), cached per lattice and cut.

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/glu_gfix.h"
#include "fft.cuh"
#include "su3_log.cuh"

namespace gfix {
void count_launches(unsigned long long n);  // gfix.cu
namespace cuts {

using su3log::log_components;

thread_local std::string t_err;

int cfail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
  return -1;
}

#define CCK(call)                                                       \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess)                                              \
      return cfail("%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                   cudaGetErrorString(e_));                             \
  } while (0)

using C2 = cx<double>;

constexpr double kTwoPi = 6.283185307179586;  // GLU's TWOPI
constexpr double kPrecTol = 3 * 1.0e-14;       // PREC_TOL, NC = 3, FP64
constexpr int kNF = 16;                        // packed fields: 4 per direction

__device__ __forceinline__ C2 cm(C2 a, C2 b) {
  return mk<double>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ---------------------------------------------------------------------
// Lie fields

// -i (a - conj(b)) / 2: the off-diagonal entry of Hermitian_proj
__device__ __forceinline__ C2 off_diag(C2 a, C2 b) {
  return mk<double>((a.y + b.y) / 2., -(a.x - b.x) / 2.);
}

// packed component k of Hermitian_proj(u)
__device__ __forceinline__ C2 lin_component(const C2 *u, int k) {
  if (k == 0) {
    const double a = u[0].y, b = u[4].y, c = u[8].y;
    return mk<double>((2 * a - b - c) / 3., (2 * b - a - c) / 3.);
  }
  if (k == 1) return off_diag(u[1], u[3]);
  if (k == 2) return off_diag(u[2], u[6]);
  return off_diag(u[5], u[7]);
}

struct CutCtx {
  int L[4];
  int V;
  const C2 *links;  // GLU's AoS links, [V][4][9]
  C2 *F;            // packed fields, [16][V]
  const C2 *tw;     // twiddle pool, exp(-2 pi i k / n) per axis
  FftAxis ax[4];
  int zt_b;         // x columns per zt tile
};

// x and y transforms of one xy plane of one packed field; LINKS: the field
// is the linear Lie field computed here from the links
template <int PT, bool ODD, bool LINKS>
__global__ void __launch_bounds__(512) k_cut_xy(CutCtx c) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ FftAxis s_ax[2];
  const int Lx = c.L[0], Ly = c.L[1], P = Lx + 1;
  C2 *A = reinterpret_cast<C2 *>(smem_raw);
  C2 *twx = A + P * Ly;
  C2 *twy = twx + Lx;
  if (threadIdx.x == 0) {
    s_ax[0] = c.ax[0];
    s_ax[1] = c.ax[1];
  }
  for (int k = threadIdx.x; k < Lx; k += blockDim.x) twx[k] = c.tw[c.ax[0].tw_off + k];
  for (int k = threadIdx.x; k < Ly; k += blockDim.x) twy[k] = c.tw[c.ax[1].tw_off + k];
  // field fastest in the grid: the 16 blocks of one plane run together and
  // share the plane's link sectors in L2
  const int f = blockIdx.x, plane = blockIdx.y;
  const int mu = f >> 2, comp = f & 3;
  const int n = Lx * Ly;
  const size_t base = (size_t)plane * n;
  const int lx_sh = log2_if_pow2(Lx);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int y = fdiv(e, Lx, lx_sh);
      C2 v;
      if constexpr (LINKS)
        v = lin_component(c.links + ((base + e) * 4 + mu) * 9, comp);
      else
        v = c.F[(size_t)f * c.V + base + e];
      A[y * P + (e - y * Lx)] = v;
    }
  }
  __syncthreads();
  const PencilMap mx = pmap(Ly, 1, 0, P, 1);
  const PencilMap my = pmap(Lx, Lx, 1, 0, P);
  smem_fft<double, PT, ODD>(A, mx, s_ax[0], twx, true);
  smem_fft<double, PT, ODD>(A, my, s_ax[1], twy, true);
  C2 *out = c.F + (size_t)f * c.V + base;
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int y = fdiv(e, Lx, lx_sh);
      out[e] = A[y * P + (e - y * Lx)];
    }
  }
}

// z and t transforms of a tile of zt_b x columns at fixed y
template <int PT, bool ODD>
__global__ void __launch_bounds__(512) k_cut_zt(CutCtx c) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ FftAxis s_ax[2];
  const int Lx = c.L[0], Ly = c.L[1], Lz = c.L[2], Lt = c.L[3];
  const int Bw = c.zt_b;
  const int TS = Lz * Bw + 1;
  C2 *A = reinterpret_cast<C2 *>(smem_raw);
  C2 *twz = A + TS * Lt;
  C2 *twt = twz + Lz;
  if (threadIdx.x == 0) {
    s_ax[0] = c.ax[2];
    s_ax[1] = c.ax[3];
  }
  for (int k = threadIdx.x; k < Lz; k += blockDim.x) twz[k] = c.tw[c.ax[2].tw_off + k];
  for (int k = threadIdx.x; k < Lt; k += blockDim.x) twt[k] = c.tw[c.ax[3].tw_off + k];
  const int nxb = Lx / Bw;
  const int xb = blockIdx.x % nxb, y = blockIdx.x / nxb;
  C2 *data = c.F + (size_t)blockIdx.y * c.V;
  const int n = Bw * Lz * Lt;
  const size_t sz = (size_t)Lx * Ly;
  const size_t base = (size_t)xb * Bw + (size_t)Lx * y;
  const int b_sh = log2_if_pow2(Bw), z_sh = log2_if_pow2(Lz);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int q = fdiv(e, Bw, b_sh), b = e - q * Bw;
      const int t = fdiv(q, Lz, z_sh), z = q - t * Lz;
      A[b + Bw * z + TS * t] = data[base + b + sz * q];
    }
  }
  __syncthreads();
  const PencilMap mz = pmap(Lt * Bw, Bw, 1, TS, Bw);
  const PencilMap mt = pmap(Lz * Bw, Lz * Bw, 1, 0, TS);
  smem_fft<double, PT, ODD>(A, mz, s_ax[0], twz, true);
  smem_fft<double, PT, ODD>(A, mt, s_ax[1], twt, true);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int q = fdiv(e, Bw, b_sh), b = e - q * Bw;
      const int t = fdiv(q, Lz, z_sh), z = q - t * Lz;
      data[base + b + sz * q] = A[b + Bw * z + TS * t];
    }
  }
}

// the same two passes with compile-time extents (the common lattices)
template <int LX, int LY, bool LINKS>
__global__ void __launch_bounds__(ct_threads(LX *LY), ct_minb(LX *LY))
    k_cut_xy_ct(CutCtx c) {
  constexpr int P = LX + 1, N = LX * LY, BD = ct_threads(N);
  constexpr int EPT = (N + BD - 1) / BD;
  extern __shared__ unsigned char smem_raw[];
  C2 *A = reinterpret_cast<C2 *>(smem_raw);
  C2 *twx = A + P * LY;
  C2 *twy = twx + LX;
  for (int k = threadIdx.x; k < LX; k += BD) twx[k] = c.tw[c.ax[0].tw_off + k];
  for (int k = threadIdx.x; k < LY; k += BD) twy[k] = c.tw[c.ax[1].tw_off + k];
  const int f = blockIdx.x, plane = blockIdx.y;
  const int mu = f >> 2, comp = f & 3;
  const size_t base = (size_t)plane * N;
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) {
      C2 v;
      if constexpr (LINKS)
        v = lin_component(c.links + ((base + e) * 4 + mu) * 9, comp);
      else
        v = c.F[(size_t)f * c.V + base + e];
      A[(e / LX) * P + e % LX] = v;
    }
  }
  __syncthreads();
  ct_stages<double, LX, 1, LY, 1, 0, P, 1, BD>(A, twx, true);   // rows
  ct_stages<double, LY, 1, LX, LX, 1, 0, P, BD>(A, twy, true);  // columns
  C2 *out = c.F + (size_t)f * c.V + base;
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) out[e] = A[(e / LX) * P + e % LX];
  }
}

template <int LZ, int LT, int B>
__global__ void __launch_bounds__(ct_threads(B *LZ *LT), ct_minb(B *LZ *LT))
    k_cut_zt_ct(CutCtx c) {
  constexpr int TS = LZ * B + zt_pad(B);  // padded t-stride
  constexpr int N = B * LZ * LT, BD = ct_threads(N);
  constexpr int EPT = (N + BD - 1) / BD;
  extern __shared__ unsigned char smem_raw[];
  C2 *A = reinterpret_cast<C2 *>(smem_raw);
  C2 *twz = A + TS * LT;
  C2 *twt = twz + LZ;
  for (int k = threadIdx.x; k < LZ; k += BD) twz[k] = c.tw[c.ax[2].tw_off + k];
  for (int k = threadIdx.x; k < LT; k += BD) twt[k] = c.tw[c.ax[3].tw_off + k];
  const int Lx = c.L[0], Ly = c.L[1];
  const int nxb = Lx / B;
  const int xb = blockIdx.x % nxb, y = blockIdx.x / nxb;
  C2 *data = c.F + (size_t)blockIdx.y * c.V;
  const size_t sz = (size_t)Lx * Ly;
  const size_t base = (size_t)xb * B + (size_t)Lx * y;
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) {
      const int q = e / B, b = e % B, t = q / LZ, z = q % LZ;
      A[b + B * z + TS * t] = data[base + b + sz * q];
    }
  }
  __syncthreads();
  ct_stages<double, LZ, 1, LT * B, B, 1, TS, B, BD>(A, twz, true);
  ct_stages<double, LT, 1, LZ * B, LZ * B, 1, 0, TS, BD>(A, twt, true);
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) {
      const int q = e / B, b = e % B, t = q / LZ, z = q % LZ;
      data[base + b + sz * q] = A[b + B * z + TS * t];
    }
  }
}

// all four packed fields of one direction of one xy plane per block: each
// thread reads whole 144-byte link records (the element pairs of a 32-byte
// sector meet in L1), and the four tiles are transformed together
template <int LX, int LY, bool LOG>
__global__ void __launch_bounds__(ct_threads(4 * LX * LY), ct_minb(4 * LX * LY))
    k_cut_xy4_ct(CutCtx c) {
  constexpr int P = LX + 1, N = LX * LY, T = P * LY, BD = ct_threads(4 * N);
  constexpr int SPT = (N + BD - 1) / BD;  // sites per thread
  constexpr int EPT = (4 * N + BD - 1) / BD;
  extern __shared__ unsigned char smem_raw[];
  C2 *A = reinterpret_cast<C2 *>(smem_raw);
  C2 *twx = A + 4 * T;
  C2 *twy = twx + LX;
  for (int k = threadIdx.x; k < LX; k += BD) twx[k] = c.tw[c.ax[0].tw_off + k];
  for (int k = threadIdx.x; k < LY; k += BD) twy[k] = c.tw[c.ax[1].tw_off + k];
  const int mu = blockIdx.x, plane = blockIdx.y;
  const size_t base = (size_t)plane * N;
#pragma unroll
  for (int k = 0; k < SPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) {
      const C2 *u = c.links + ((base + e) * 4 + mu) * 9;
      C2 r[9];
#pragma unroll
      for (int j = 0; j < 9; j++) r[j] = u[j];
      const int o = (e / LX) * P + e % LX;
      if constexpr (LOG) {
        C2 q4[4];
        log_components(r, q4);
#pragma unroll
        for (int q = 0; q < 4; q++) A[q * T + o] = q4[q];
      } else {
#pragma unroll
        for (int q = 0; q < 4; q++) A[q * T + o] = lin_component(r, q);
      }
    }
  }
  __syncthreads();
  ct_stages<double, LX, 1, 4 * LY, 1, 0, P, 1, BD>(A, twx, true);       // rows
  ct_stages<double, LY, 1, 4 * LX, LX, 1, T, P, BD>(A, twy, true);      // columns
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if ((4 * N) % BD == 0 || e < 4 * N) {
      const int q = e / N, r = e % N;
      c.F[(size_t)(mu * 4 + q) * c.V + base + r] = A[q * T + (r / LX) * P + r % LX];
    }
  }
}

// the logarithmic Lie fields packed into F, one thread per site and
// direction (for the per-field xy passes)
__global__ void __launch_bounds__(128) k_cut_log_pack(CutCtx c) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)c.V * 4) return;
  const size_t site = t >> 2;
  const int mu = (int)(t & 3);
  C2 r[9];
  const C2 *u = c.links + t * 9;
#pragma unroll
  for (int j = 0; j < 9; j++) r[j] = u[j];
  C2 q4[4];
  log_components(r, q4);
#pragma unroll
  for (int q = 0; q < 4; q++) c.F[(size_t)(mu * 4 + q) * c.V + site] = q4[q];
}

using CutFn = void (*)(CutCtx);

static CutFn xy4_ct(int lx, int ly, bool log) {
#define GFIX_CXY4(n) \
  if (lx == n && ly == n) return log ? k_cut_xy4_ct<n, n, true> : k_cut_xy4_ct<n, n, false>;
  GFIX_CXY4(8) GFIX_CXY4(16) GFIX_CXY4(24) GFIX_CXY4(32) GFIX_CXY4(48)
#undef GFIX_CXY4
  return nullptr;
}

static CutFn xy_ct(int lx, int ly, bool links) {
#define GFIX_CXY(n) \
  if (lx == n && ly == n) return links ? k_cut_xy_ct<n, n, true> : k_cut_xy_ct<n, n, false>;
  GFIX_CXY(8) GFIX_CXY(16) GFIX_CXY(24) GFIX_CXY(32) GFIX_CXY(48) GFIX_CXY(64)
#undef GFIX_CXY
  return nullptr;
}

// compiled zt passes of (Lz, Lt): (tile width, kernel) candidates; the
// width only regroups pencils, so every candidate gives the same bits
static std::vector<std::pair<int, CutFn>> zt_ct(int lz, int lt, int lx) {
  std::vector<std::pair<int, CutFn>> v;
#define GFIX_CZT(z, t, bb) \
  if (lz == z && lt == t && lx % bb == 0) v.push_back({bb, k_cut_zt_ct<z, t, bb>});
  GFIX_CZT(8, 8, 8) GFIX_CZT(8, 16, 4) GFIX_CZT(16, 16, 4) GFIX_CZT(16, 32, 2)
  GFIX_CZT(16, 32, 4) GFIX_CZT(24, 48, 1) GFIX_CZT(24, 48, 2) GFIX_CZT(32, 32, 2)
  GFIX_CZT(32, 32, 4) GFIX_CZT(32, 64, 1) GFIX_CZT(32, 64, 2) GFIX_CZT(32, 64, 4)
  GFIX_CZT(48, 96, 1) GFIX_CZT(48, 96, 2) GFIX_CZT(64, 128, 1)
#undef GFIX_CZT
  return v;
}

// per listed momentum i: G[i][mu][9] = A_mu(p) e^{i p_mu / 2} and the
// p-space error term |sum_mu,j p_mu G_mu,j| / 9 (pspace_landau.c:38-77)
__global__ void __launch_bounds__(128) k_cut_gather(const C2 *F, int V, int nmom,
                                                    const int2 *sites,
                                                    const C2 *phase,
                                                    const double *pmu, C2 *G,
                                                    double *err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmom) return;
  const int2 st = sites[i];
  C2 sum = mk<double>(0., 0.);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const C2 *f = F + (size_t)(mu * 4) * V;
    const C2 c0p = f[st.x], c0n = f[st.y];
    const C2 c1p = f[(size_t)V + st.x], c1n = f[(size_t)V + st.y];
    const C2 c2p = f[2 * (size_t)V + st.x], c2n = f[2 * (size_t)V + st.y];
    const C2 c3p = f[3 * (size_t)V + st.x], c3n = f[3 * (size_t)V + st.y];
    C2 q[9];
    q[0] = mk<double>((c0p.x + c0n.x) / 2., (c0p.y - c0n.y) / 2.);
    q[4] = mk<double>((c0p.y + c0n.y) / 2., -(c0p.x - c0n.x) / 2.);
    q[8] = mk<double>(-(q[0].x + q[4].x), -(q[0].y + q[4].y));
    q[1] = c1p;
    q[2] = c2p;
    q[5] = c3p;
    q[3] = mk<double>(c1n.x, -c1n.y);
    q[6] = mk<double>(c2n.x, -c2n.y);
    q[7] = mk<double>(c3n.x, -c3n.y);
    const C2 ph = phase[i * 4 + mu];
    const double p = pmu[i * 4 + mu];
    C2 *g = G + ((size_t)i * 4 + mu) * 9;
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const C2 v = cm(q[j], ph);
      g[j] = v;
      sum.x += v.x * p;
      sum.y += v.y * p;
    }
  }
  err[i] = hypot(sum.x, sum.y) / 9.;
}

// tr(a b)
__device__ __forceinline__ C2 tr_ab(const C2 *a, const C2 *b) {
  C2 t = mk<double>(0., 0.);
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const C2 v = cm(a[r * 3 + s], b[s * 3 + r]);
      t.x += v.x;
      t.y += v.y;
    }
  return t;
}

__device__ __forceinline__ void mat_mul(C2 *o, const C2 *a, const C2 *b) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int s = 0; s < 3; s++) {
      C2 t = mk<double>(0., 0.);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const C2 v = cm(a[r * 3 + k], b[k * 3 + s]);
        t.x += v.x;
        t.y += v.y;
      }
      o[r * 3 + s] = t;
    }
}

struct Norms {
  double g2, g0, gl, g3;  // glueprop.c:92-94, MOMgg.c:165-168
};

// transverse and longitudinal propagators (glueprop.c:66-86) for the first
// half of the list and the zero momentum; the host mirrors the rest
__global__ void __launch_bounds__(128) k_cut_props(const C2 *G, int zero,
                                                   const double *pmu,
                                                   const double *psq, Norms nm,
                                                   double *tr_out,
                                                   double *lo_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > zero) return;
  const C2 *g = G + (size_t)i * 36;
  const double spsq = 1.0 / psq[i];
  double T = 0.0, Lg = 0.0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
      double re = 0.0;
#pragma unroll
      for (int j = 0; j < 9; j++) {
        const C2 a = g[mu * 9 + j], b = g[nu * 9 + j];
        re += a.x * b.x + a.y * b.y;
      }
      const double common = pmu[i * 4 + mu] * pmu[i * 4 + nu] * spsq * re;
      T += (mu != nu) ? -common : re - common;
      Lg += common;
    }
  tr_out[i] = T * (i == zero ? nm.g0 : nm.g2);
  lo_out[i] = Lg * nm.gl;
}

// MOMgg two- and three-point functions (MOMgg.c:89-120, 170-206)
__global__ void __launch_bounds__(128) k_cut_momgg(const C2 *G, int nmom,
                                                   const double *pmu,
                                                   const double *psq, Norms nm,
                                                   double *g2_out,
                                                   double *g3_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmom) return;
  const int zp = (nmom - 1) / 2;
  const C2 *gp = G + (size_t)i * 36;
  const C2 *gc = G + (size_t)(nmom - 1 - i) * 36;
  const C2 *g0 = G + (size_t)zp * 36;
  double t2 = 0.0;
  for (int mu = 0; mu < 4; mu++) t2 += tr_ab(gp + mu * 9, gc + mu * 9).x;
  g2_out[i] = t2 * (i == zp ? nm.g0 : nm.g2);
  const double sp = psq[i];
  C2 AA[9], Ar[9], AP[9], AM[9], tmp[9];
#pragma unroll
  for (int j = 0; j < 9; j++) AA[j] = Ar[j] = AP[j] = AM[j] = mk<double>(0., 0.);
  for (int mu = 0; mu < 4; mu++) {
    const double m = pmu[i * 4 + mu];
    mat_mul(tmp, gp + mu * 9, gc + mu * 9);
#pragma unroll
    for (int j = 0; j < 9; j++) {
      AA[j].x += tmp[j].x;
      AA[j].y += tmp[j].y;
      Ar[j].x += m * g0[mu * 9 + j].x;
      Ar[j].y += m * g0[mu * 9 + j].y;
      AP[j].x += m * gp[mu * 9 + j].x;
      AP[j].y += m * gp[mu * 9 + j].y;
      const double s = -m / sp;
      AM[j].x += s * gc[mu * 9 + j].x;
      AM[j].y += s * gc[mu * 9 + j].y;
    }
  }
  const C2 trans = tr_ab(AA, Ar);
  mat_mul(tmp, Ar, AP);
  const C2 wiv = tr_ab(tmp, AM);
  g3_out[i] = ((trans.x + wiv.x) / sp) * nm.g3;
}

// ---------------------------------------------------------------------
// momentum list (src/Cuts/cut_routines.c)

struct CutKey {
  int dir, type;
  size_t max_mom, angle;
  double cyl_width;
  bool operator<(const CutKey &o) const {
    return std::tie(dir, type, max_mom, angle, cyl_width) <
           std::tie(o.dir, o.type, o.max_mom, o.angle, o.cyl_width);
  }
};

struct MomList {
  std::vector<int> mom;     // 4 per momentum, -pi..pi zone
  std::vector<int2> sites;  // 0..2pi-zone sites of p and -p
  std::vector<C2> phase;    // e^{i p_mu / 2} per momentum and direction
  std::vector<double> pmu;  // 2 sin(p_mu / 2)
  std::vector<double> psq;  // sum_mu pmu^2, 1 below PREC_TOL
  size_t n() const { return sites.size(); }
};

// body diagonal d of the hypercube: component mu is +1 where bit mu of d
// is set, else -1 (get_diagonal)
static void diagonal(int d, double x[4]) {
  for (int mu = 0; mu < 4; mu++) x[mu] = ((d >> mu) & 1) ? 1.0 : -1.0;
}

// distance of q from the nearest body diagonal (cylinder_DF)
static bool cylinder_df(const double q[4], double width) {
  const double norm = 1. / (2. * std::sqrt(4));
  double x[4];
  for (int d = 0; d < 16; d++) {
    diagonal(d, x);
    double sp = 0.;
    for (int nu = 0; nu < 4; nu++) sp += q[nu] * x[nu];
    sp *= norm;
    double mod = 0.0;
    for (int nu = 0; nu < 4; nu++) {
      const double t = q[nu] - sp * x[nu];
      mod += t * t;
    }
    if (std::sqrt(mod) <= width) return true;
  }
  return false;
}

// cylinder plus cone about the body diagonals (cylinder_CJD)
static bool cylinder_cjd(const double q[4], double width, double arc) {
  double qn = 0.;
  for (int mu = 0; mu < 4; mu++) qn += q[mu] * q[mu];
  if (qn < kPrecTol) return true;
  qn = 1.0 / std::sqrt(qn);
  double x[4];
  for (int d = 0; d < 16; d++) {
    diagonal(d, x);
    double nn = 0.;
    for (int nu = 0; nu < 4; nu++) nn += x[nu] * x[nu];
    nn = qn / std::sqrt(nn);
    double sp = 0.;
    for (int nu = 0; nu < 4; nu++) sp += q[nu] * x[nu] * nn;
    const double theta = std::acos(sp);
    const double dq = std::sin(theta) / qn;
    if (dq <= width && theta <= arc * 0.01745329251994330) return true;
  }
  return false;
}

static int build_list(const int L[4], const gfix_cut_info &ci, MomList &ml) {
  int type = ci.type;
  if (ci.dir == GFIX_CUT_NONEXCEPTIONAL) type = GFIX_CUT_PSQ;
  int small = L[0];
  for (int mu = 1; mu < 4; mu++) small = std::min(small, L[mu]);
  double rats[4], tw[4];
  for (int mu = 0; mu < 4; mu++) {
    rats[mu] = (double)small / (double)L[mu];
    tw[mu] = kTwoPi / (double)L[mu];
  }
  const double width = kTwoPi * ci.cyl_width / small;
  const double maxm = (double)ci.max_mom;
  const double root = std::sqrt((double)ci.max_mom);
  // every kept momentum has (rats n_mu)^2 <= max_mom in each direction, so
  // the lexicographic scan can skip the rest of each axis
  int lo[4], hi[4];
  for (int mu = 0; mu < 4; mu++) {
    lo[mu] = -(L[mu] / 2);
    hi[mu] = L[mu] - L[mu] / 2 - 1;
    const int b = (int)std::floor(std::sqrt(maxm) / rats[mu]) + 1;
    lo[mu] = std::max(lo[mu], -b);
    hi[mu] = std::min(hi[mu], b);
  }
  ml = MomList();
  int n[4];
  for (n[3] = lo[3]; n[3] <= hi[3]; n[3]++)
    for (n[2] = lo[2]; n[2] <= hi[2]; n[2]++)
      for (n[1] = lo[1]; n[1] <= hi[1]; n[1]++)
        for (n[0] = lo[0]; n[0] <= hi[0]; n[0]++) {
          double psq = 0.;
          for (int mu = 0; mu < 4; mu++) {
            const double t = rats[mu] * n[mu];
            psq += t * t;
          }
          bool ok;
          if (type == GFIX_CUT_HYPERCUBIC) {
            ok = true;
            for (int mu = 0; mu < 4; mu++)
              if (!(std::fabs((double)n[mu] * rats[mu]) <= root)) ok = false;
          } else if (type == GFIX_CUT_CYLINDER || type == GFIX_CUT_CONICAL) {
            ok = psq <= maxm;
            if (ok) {
              double q[4];
              for (int mu = 0; mu < 4; mu++)
                q[mu] = 2. * std::sin(n[mu] * tw[mu] * 0.5);
              ok = type == GFIX_CUT_CYLINDER
                       ? cylinder_df(q, width)
                       : cylinder_cjd(q, width, (double)ci.angle);
            }
          } else {
            ok = psq <= maxm;
          }
          if (!ok) continue;
          int sp = 0, sn = 0;
          for (int mu = 3; mu >= 0; mu--) {
            const int a = n[mu] < 0 ? n[mu] + L[mu] : n[mu];
            const int b = ((-n[mu]) % L[mu] + L[mu]) % L[mu];
            sp = sp * L[mu] + a;
            sn = sn * L[mu] + b;
          }
          double ps = 0.;
          for (int mu = 0; mu < 4; mu++) {
            ml.mom.push_back(n[mu]);
            const double cache = 0.5 * n[mu] * tw[mu];
            const double p = 2.0 * std::sin(cache);
            ml.phase.push_back(mk<double>(std::cos(cache), 0.5 * p));
            const double m = 2.0 * std::sin(n[mu] * tw[mu] * 0.5);
            ml.pmu.push_back(m);
            ps += m * m;
          }
          ml.psq.push_back(ps < kPrecTol ? 1.0 : ps);
          ml.sites.push_back(make_int2(sp, sn));
        }
  return 0;
}

// ---------------------------------------------------------------------
// workspace per lattice shape

struct Work {
  int L[4] = {0, 0, 0, 0};
  int V = 0;
  cudaStream_t s = nullptr;
  CutCtx c{};
  C2 *d_links = nullptr, *d_F = nullptr, *d_tw = nullptr, *d_G = nullptr,
     *d_phase = nullptr;
  double *d_pmu = nullptr, *d_psq = nullptr, *d_err = nullptr, *d_o0 = nullptr,
         *d_o1 = nullptr;
  int2 *d_sites = nullptr;
  size_t cap = 0;  // momenta the list buffers hold
  int pt_xy = 8, pt_zt = 8, bd_xy = 128, bd_zt = 128;
  size_t sm_xy = 0, sm_zt = 0;
  bool odd = false;
  // compile-time passes, if any: xy_fn[definition] (LINEAR, LOG)
  CutFn xy_fn[2] = {nullptr, nullptr}, zt_fn = nullptr;
  bool xy4 = false;  // xy_fn are k_cut_xy4_ct (the Lie fields computed inside)
  std::map<CutKey, MomList> lists;
  const MomList *cur = nullptr;  // list on the device

  ~Work() {
    cudaFree(d_links);
    cudaFree(d_F);
    cudaFree(d_tw);
    cudaFree(d_G);
    cudaFree(d_phase);
    cudaFree(d_pmu);
    cudaFree(d_psq);
    cudaFree(d_err);
    cudaFree(d_o0);
    cudaFree(d_o1);
    cudaFree(d_sites);
    if (s) cudaStreamDestroy(s);
  }

  static size_t threads(size_t n, int pt) {
    const size_t t = (n + pt - 1) / pt;
    return std::max<size_t>(128, (t + 31) / 32 * 32);
  }

  int init(const size_t *d) {
    size_t Vs = 1;
    for (int i = 0; i < 4; i++) {
      if (d[i] < 2 || d[i] > 4096) return cfail("extent %zu outside 2..4096", d[i]);
      L[i] = (int)d[i];
      Vs *= d[i];
    }
    if (Vs > (size_t)INT32_MAX / 4) return cfail("lattice volume %zu too large", Vs);
    V = (int)Vs;
    for (int i = 0; i < 4; i++) {
      if (factorize(L[i], c.ax[i]) != 0)
        return cfail("extent %d has a prime factor above %d", L[i], kMaxRadix);
      if (L[i] % 5 == 0 || L[i] % 7 == 0) odd = true;
    }
    const size_t nxy = (size_t)L[0] * L[1];
    if (nxy > 8192) return cfail("xy plane of %zu sites above 8192", nxy);
    pt_xy = (nxy <= 4096 && !odd) ? 8 : 16;
    bd_xy = (int)threads(nxy, pt_xy);
    sm_xy = ((size_t)(L[0] + 1) * L[1] + L[0] + L[1]) * sizeof(C2);
    const size_t nzt = (size_t)L[2] * L[3];
    if (nzt > 8192) return cfail("zt column of %zu sites above 8192", nzt);
    int b = 1;
    while (L[0] % (2 * b) == 0 && 2 * b * nzt <= 4096) b *= 2;
    c.zt_b = b;
    pt_zt = (b * nzt <= 4096 && !odd) ? 8 : 16;
    bd_zt = (int)threads(b * nzt, pt_zt);
    sm_zt = ((size_t)(L[2] * b + 1) * L[3] + L[2] + L[3]) * sizeof(C2);
    CCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    // compile-time passes where the extents have them
    if (!odd) {
      const size_t sm4 = (4 * (size_t)(L[0] + 1) * L[1] + L[0] + L[1]) * sizeof(C2);
      if (xy4_ct(L[0], L[1], false) && sm4 <= 200u * 1024u) {
        xy4 = true;
        xy_fn[0] = xy4_ct(L[0], L[1], false);
        xy_fn[1] = xy4_ct(L[0], L[1], true);
        bd_xy = ct_threads(4 * L[0] * L[1]);
        sm_xy = sm4;
      } else if (xy_ct(L[0], L[1], true)) {
        xy_fn[0] = xy_ct(L[0], L[1], true);
        xy_fn[1] = xy_ct(L[0], L[1], false);  // on the packed logarithms
        bd_xy = ct_threads(L[0] * L[1]);
      }
    }
    std::vector<C2> tw;
    for (int a = 0; a < 4; a++) {
      c.ax[a].tw_off = (int)tw.size();
      for (int k = 0; k < L[a]; k++) {
        const double ang = 6.283185307179586476925286766559 * k / L[a];
        tw.push_back(mk<double>(std::cos(ang), -std::sin(ang)));
      }
    }
    CCK(cudaMalloc(&d_tw, tw.size() * sizeof(C2)));
    CCK(cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(C2), cudaMemcpyHostToDevice));
    CCK(cudaMalloc(&d_F, (size_t)kNF * V * sizeof(C2)));
    for (int i = 0; i < 4; i++) c.L[i] = L[i];
    c.V = V;
    c.tw = d_tw;
    c.F = d_F;
    if (set_attrs()) return -1;
    return odd ? 0 : pick_zt();
  }

  // the fastest compiled zt pass for this shape (timed once on zeroed
  // fields; all candidates give identical results)
  int pick_zt() {
    const auto cands = zt_ct(L[2], L[3], L[0]);
    if (cands.empty()) return 0;
    CCK(cudaMemsetAsync(d_F, 0, (size_t)kNF * V * sizeof(C2), s));
    cudaEvent_t a, b;
    CCK(cudaEventCreate(&a));
    CCK(cudaEventCreate(&b));
    float best = 1e30f;
    for (const auto &cd : cands) {
      const int bw = cd.first;
      const size_t sm = ((size_t)(L[2] * bw + zt_pad(bw)) * L[3] + L[2] + L[3]) * sizeof(C2);
      if (sm > 200u * 1024u || attr(cd.second, sm)) continue;
      CutCtx cc = c;
      cc.zt_b = bw;
      const int bd = ct_threads(bw * L[2] * L[3]);
      const dim3 g((L[0] / bw) * L[1], kNF);
      cd.second<<<g, bd, sm, s>>>(cc);
      CCK(cudaEventRecord(a, s));
      for (int r = 0; r < 3; r++) cd.second<<<g, bd, sm, s>>>(cc);
      CCK(cudaEventRecord(b, s));
      CCK(cudaEventSynchronize(b));
      float ms = 0.f;
      CCK(cudaEventElapsedTime(&ms, a, b));
      if (ms < best) {
        best = ms;
        zt_fn = cd.second;
        c.zt_b = bw;
        bd_zt = bd;
        sm_zt = sm;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CCK(cudaGetLastError());
    return 0;
  }

  template <typename K>
  int attr(K k, size_t sm) {
    CCK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    return 0;
  }
  int set_attrs() {
    if (attr(k_cut_xy<8, false, true>, sm_xy) || attr(k_cut_xy<16, false, true>, sm_xy) ||
        attr(k_cut_xy<16, true, true>, sm_xy) || attr(k_cut_xy<8, false, false>, sm_xy) ||
        attr(k_cut_xy<16, false, false>, sm_xy) || attr(k_cut_xy<16, true, false>, sm_xy) ||
        attr(k_cut_zt<8, false>, sm_zt) || attr(k_cut_zt<16, false>, sm_zt) ||
        attr(k_cut_zt<16, true>, sm_zt))
      return -1;
    for (CutFn f : xy_fn)
      if (f && attr(f, sm_xy)) return -1;
    return 0;
  }

  const MomList *list(const gfix_cut_info &ci) {
    const CutKey k{ci.dir, ci.type, ci.max_mom, ci.angle, ci.cyl_width};
    auto it = lists.find(k);
    if (it != lists.end()) return &it->second;
    MomList ml;
    if (build_list(L, ci, ml)) return nullptr;
    return &lists.emplace(k, std::move(ml)).first->second;
  }

  int upload(const MomList *ml) {
    if (cur == ml) return 0;
    const size_t n = std::max<size_t>(ml->n(), 1);
    if (n > cap) {
      cudaFree(d_G);
      cudaFree(d_phase);
      cudaFree(d_pmu);
      cudaFree(d_psq);
      cudaFree(d_err);
      cudaFree(d_o0);
      cudaFree(d_o1);
      cudaFree(d_sites);
      d_G = d_phase = nullptr;
      d_pmu = d_psq = d_err = d_o0 = d_o1 = nullptr;
      d_sites = nullptr;
      cap = 0;
      CCK(cudaMalloc(&d_G, n * 36 * sizeof(C2)));
      CCK(cudaMalloc(&d_phase, n * 4 * sizeof(C2)));
      CCK(cudaMalloc(&d_pmu, n * 4 * sizeof(double)));
      CCK(cudaMalloc(&d_psq, n * sizeof(double)));
      CCK(cudaMalloc(&d_err, n * sizeof(double)));
      CCK(cudaMalloc(&d_o0, n * sizeof(double)));
      CCK(cudaMalloc(&d_o1, n * sizeof(double)));
      CCK(cudaMalloc(&d_sites, n * sizeof(int2)));
      cap = n;
    }
    cur = nullptr;
    if (ml->n()) {
      CCK(cudaMemcpyAsync(d_phase, ml->phase.data(), ml->n() * 4 * sizeof(C2),
                          cudaMemcpyHostToDevice, s));
      CCK(cudaMemcpyAsync(d_pmu, ml->pmu.data(), ml->n() * 4 * sizeof(double),
                          cudaMemcpyHostToDevice, s));
      CCK(cudaMemcpyAsync(d_psq, ml->psq.data(), ml->n() * sizeof(double),
                          cudaMemcpyHostToDevice, s));
      CCK(cudaMemcpyAsync(d_sites, ml->sites.data(), ml->n() * sizeof(int2),
                          cudaMemcpyHostToDevice, s));
    }
    CCK(cudaStreamSynchronize(s));
    cur = ml;
    return 0;
  }

  int ensure_links() {
    if (!d_links) CCK(cudaMalloc(&d_links, (size_t)V * 36 * sizeof(C2)));
    return 0;
  }

  // the transforms of the Lie fields (definition def) of c.links into
  // d_F; `mid` (may be null) is recorded between the xy and the zt pass
  void transform(int def, cudaEvent_t mid = nullptr) {
    const bool log = def == GFIX_FIELD_LOG;
    const dim3 gxy(xy4 ? 4 : kNF, L[2] * L[3]);
    if (log && !xy4) {
      k_cut_log_pack<<<(unsigned)(((size_t)V * 4 + 127) / 128), 128, 0, s>>>(c);
      count_launches(1);
    }
    if (xy_fn[log])
      xy_fn[log]<<<gxy, bd_xy, sm_xy, s>>>(c);
    else if (odd)
      log ? k_cut_xy<16, true, false><<<gxy, bd_xy, sm_xy, s>>>(c)
          : k_cut_xy<16, true, true><<<gxy, bd_xy, sm_xy, s>>>(c);
    else if (pt_xy == 8)
      log ? k_cut_xy<8, false, false><<<gxy, bd_xy, sm_xy, s>>>(c)
          : k_cut_xy<8, false, true><<<gxy, bd_xy, sm_xy, s>>>(c);
    else
      log ? k_cut_xy<16, false, false><<<gxy, bd_xy, sm_xy, s>>>(c)
          : k_cut_xy<16, false, true><<<gxy, bd_xy, sm_xy, s>>>(c);
    if (mid) cudaEventRecord(mid, s);
    const dim3 gzt((L[0] / c.zt_b) * L[1], kNF);
    if (zt_fn)
      zt_fn<<<gzt, bd_zt, sm_zt, s>>>(c);
    else if (odd)
      k_cut_zt<16, true><<<gzt, bd_zt, sm_zt, s>>>(c);
    else if (pt_zt == 8)
      k_cut_zt<8, false><<<gzt, bd_zt, sm_zt, s>>>(c);
    else
      k_cut_zt<16, false><<<gzt, bd_zt, sm_zt, s>>>(c);
    count_launches(2);
  }

  Norms norms() const {
    const double Vd = (double)V;
    return Norms{2.0 / ((9 - 1) * (4 - 1) * Vd), 2.0 / ((9 - 1) * (4) * Vd),
                 2.0 / ((9 - 1) * Vd), 4.0 / (2.0 * 3 * (9 - 1) * (4 - 1) * Vd)};
  }

  // gather and contract on the device list
  void measure(int dir) {
    const int n = (int)cur->n();
    if (n == 0) return;
    const int nb = (n + 127) / 128;
    k_cut_gather<<<nb, 128, 0, s>>>(d_F, V, n, d_sites, d_phase, d_pmu, d_G, d_err);
    if (dir == GFIX_CUT_GLUON_PROPS)
      k_cut_props<<<nb, 128, 0, s>>>(d_G, n >> 1, d_pmu, d_psq, norms(), d_o0, d_o1);
    else if (dir == GFIX_CUT_EXCEPTIONAL)
      k_cut_momgg<<<nb, 128, 0, s>>>(d_G, n, d_pmu, d_psq, norms(), d_o0, d_o1);
    count_launches(dir == GFIX_CUT_FIELDS ? 1 : 2);
  }

  // results to the host, as GLU fills them
  int fetch(int dir, double *out0, double *out1, double *perr) {
    const size_t n = cur->n();
    std::vector<double> err(n);
    if (n) CCK(cudaMemcpyAsync(err.data(), d_err, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dir == GFIX_CUT_FIELDS) {
      if (out0 && n)
        CCK(cudaMemcpyAsync(out0, d_G, n * 36 * sizeof(C2), cudaMemcpyDeviceToHost, s));
    } else if (n) {
      if (out0) CCK(cudaMemcpyAsync(out0, d_o0, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (out1) CCK(cudaMemcpyAsync(out1, d_o1, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CCK(cudaStreamSynchronize(s));
    CCK(cudaGetLastError());
    if (dir == GFIX_CUT_GLUON_PROPS) {
      // p, -p symmetry of the list (glueprop.c:128-132)
      const size_t zero = n >> 1;
      for (size_t i = zero + 1; i < n; i++) {
        if (out0) out0[i] = out0[n - i - 1];
        if (out1) out1[i] = out1[n - i - 1];
      }
    }
    if (perr) {
      double e = 0.0;
      for (size_t i = 0; i < n; i++) e += err[i];
      *perr = n ? e / (double)n : 0.0;
    }
    return 0;
  }
};

// one workspace per (device, lattice shape): a workspace's buffers and
// stream belong to the device that was current when it was made
static std::map<std::array<size_t, 5>, std::unique_ptr<Work>> g_work;
static std::mutex g_work_mu;

static Work *work_for(const size_t *dims) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cfail("no CUDA device");
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

static int check_info(const size_t *dims, const gfix_cut_info *ci) {
  if (!dims || !ci) return cfail("null dims or cut info");
  if (ci->dir != GFIX_CUT_GLUON_PROPS && ci->dir != GFIX_CUT_EXCEPTIONAL &&
      ci->dir != GFIX_CUT_FIELDS)
    return cfail("cut mode %d not supported (GLUON_PROPS, EXCEPTIONAL, FIELDS)", ci->dir);
  if (ci->type < GFIX_CUT_HYPERCUBIC || ci->type > GFIX_CUT_CONICAL)
    return cfail("momentum cut type %d unknown", ci->type);
  if (ci->definition != GFIX_FIELD_LINEAR && ci->definition != GFIX_FIELD_LOG)
    return cfail("field definition %d unknown", ci->definition);
  return 0;
}

// the whole measurement on links already on the device (GLU's AoS layout)
static int run(Work *w, const gfix_cut_info *ci, size_t nmom, double *out0,
               double *out1, double *perr) {
  const MomList *ml = w->list(*ci);
  if (!ml) return -1;
  if (nmom != ml->n())
    return cfail("%zu momenta given, the cut keeps %zu", nmom, ml->n());
  if (w->upload(ml)) return -1;
  w->transform(ci->definition);
  w->measure(ci->dir);
  CCK(cudaGetLastError());
  return w->fetch(ci->dir, out0, out1, perr);
}

// ---------------------------------------------------------------------
// GLU's output file (cut_output.c)

static void put_be32(std::vector<unsigned char> &b, uint32_t v) {
  for (int k = 3; k >= 0; k--) b.push_back((unsigned char)(v >> (8 * k)));
}
static void put_be64(std::vector<unsigned char> &b, double d) {
  uint64_t v;
  memcpy(&v, &d, 8);
  for (int k = 7; k >= 0; k--) b.push_back((unsigned char)(v >> (8 * k)));
}

// output_str_struct (cut_output.c:121-242) for these modes
static std::string output_name(const size_t *dims, const gfix_cut_info &ci,
                               const char *where, size_t flow) {
  std::string s = where ? where : "./";
  s += ci.dir == GFIX_CUT_GLUON_PROPS ? "G2F2" : ci.dir == GFIX_CUT_FIELDS ? "MATS" : "MOMgg";
  char tmp[256];
  snprintf(tmp, sizeof tmp, "_SU3_%zux%zux%zux%zu_%zu_", dims[0], dims[1], dims[2],
           dims[3], ci.max_mom);
  s += tmp;
  switch (ci.type) {
    case GFIX_CUT_HYPERCUBIC: s += "cutHYP"; break;
    case GFIX_CUT_PSQ: s += "cutPSQ"; break;
    case GFIX_CUT_CYLINDER:
      snprintf(tmp, sizeof tmp, "cutCYL_w%g", ci.cyl_width);
      s += tmp;
      break;
    default:
      snprintf(tmp, sizeof tmp, "cutCON_%zu", ci.angle);
      s += tmp;
  }
  s += "_SINMOM";
  s += ci.definition == GFIX_FIELD_LOG ? "_LOG" : "_LIN";
  snprintf(tmp, sizeof tmp, ".%zu.bin", flow);
  s += tmp;
  return s;
}

static int write_file(const std::string &path, const MomList &ml, int dir,
                      const std::vector<double> &o0, const std::vector<double> &o1) {
  std::vector<unsigned char> b;
  const size_t n = ml.n();
  b.reserve(8 + n * 20 + 16 + n * 8 * (dir == GFIX_CUT_FIELDS ? 72 : 2));
  // write_mom_veclist: count, then (4, p0, p1, p2, p3) per momentum
  put_be32(b, (uint32_t)n);
  for (size_t i = 0; i < n; i++) {
    put_be32(b, 4u);
    for (int mu = 0; mu < 4; mu++) put_be32(b, (uint32_t)ml.mom[i * 4 + mu]);
  }
  put_be32(b, (uint32_t)n);
  if (dir == GFIX_CUT_FIELDS) {  // write_lattice_fields
    for (size_t k = 0; k < n * 72; k++) put_be64(b, o0[k]);
  } else {  // write_g2g3_to_list
    for (size_t k = 0; k < n; k++) put_be64(b, o0[k]);
    put_be32(b, (uint32_t)n);
    for (size_t k = 0; k < n; k++) put_be64(b, o1[k]);
  }
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return cfail("cannot open %s for writing", path.c_str());
  const size_t wr = fwrite(b.data(), 1, b.size(), f);
  fclose(f);
  if (wr != b.size()) return cfail("short write to %s", path.c_str());
  return 0;
}

}  // namespace cuts
}  // namespace gfix

using namespace gfix::cuts;

extern "C" {

const char *gfix_cuts_error(void) { return t_err.c_str(); }

long gfix_cut_veclist(const size_t dims[4], const gfix_cut_info *ci, int32_t *mom,
                      size_t cap) {
  if (!dims || !ci) return cfail("null dims or cut info");
  int L[4];
  for (int i = 0; i < 4; i++) {
    if (dims[i] < 2 || dims[i] > 4096) return cfail("extent %zu outside 2..4096", dims[i]);
    L[i] = (int)dims[i];
  }
  MomList ml;
  if (build_list(L, *ci, ml)) return -1;
  if (mom)
    for (size_t i = 0; i < ml.n() && i < cap; i++)
      for (int mu = 0; mu < 4; mu++) mom[i * 4 + mu] = ml.mom[i * 4 + mu];
  return (long)ml.n();
}

int gfix_cuts_measure_device(const double *d_links, const size_t dims[4],
                             const gfix_cut_info *ci, size_t nmom, double *out0,
                             double *out1, double *pspace_err) {
  if (!d_links) return cfail("null links");
  if (check_info(dims, ci)) return -1;
  Work *w = work_for(dims);
  if (!w) return -1;
  // the library's stream does not synchronise with the caller's: wait for
  // all work on the device before the links are read
  CCK(cudaDeviceSynchronize());
  w->c.links = reinterpret_cast<const C2 *>(d_links);
  return run(w, ci, nmom, out0, out1, pspace_err);
}

int gfix_cuts_measure(const double *links, const size_t dims[4], const gfix_cut_info *ci,
                      size_t nmom, double *out0, double *out1, double *pspace_err) {
  if (!links) return cfail("null links");
  if (check_info(dims, ci)) return -1;
  Work *w = work_for(dims);
  if (!w || w->ensure_links()) return -1;
  CCK(cudaMemcpyAsync(w->d_links, links, (size_t)w->V * 36 * sizeof(C2),
                      cudaMemcpyHostToDevice, w->s));
  w->c.links = w->d_links;
  return run(w, ci, nmom, out0, out1, pspace_err);
}

int gfix_cuts_write(const double *links, const size_t dims[4], const gfix_cut_info *ci,
                    const char *where, size_t flow, double *pspace_err, char *path_out,
                    size_t path_cap) {
  if (check_info(dims, ci)) return -1;
  Work *w = work_for(dims);
  if (!w) return -1;
  const MomList *ml = w->list(*ci);
  if (!ml) return -1;
  if (ml->n() == 0) return cfail("empty momentum list");
  const size_t n = ml->n();
  std::vector<double> o0(ci->dir == GFIX_CUT_FIELDS ? n * 72 : n), o1(n);
  double e = 0.0;
  if (gfix_cuts_measure(links, dims, ci, n, o0.data(), o1.data(), &e)) return -1;
  if (pspace_err) *pspace_err = e;
  const std::string path = output_name(dims, *ci, where, flow);
  if (path_out && path_cap) snprintf(path_out, path_cap, "%s", path.c_str());
  return write_file(path, *ml, ci->dir, o0, o1);
}

int gfix_profile_cuts(const double *d_links, const size_t dims[4], const gfix_cut_info *ci,
                      int reps, float ms[3]) {
  if (!d_links || !ms || reps < 1) return cfail("bad arguments to gfix_profile_cuts");
  if (check_info(dims, ci)) return -1;
  Work *w = work_for(dims);
  if (!w) return -1;
  CCK(cudaDeviceSynchronize());
  w->c.links = reinterpret_cast<const C2 *>(d_links);
  const MomList *ml = w->list(*ci);
  if (!ml || w->upload(ml)) return -1;
  cudaEvent_t ev[4];
  for (auto &e : ev) CCK(cudaEventCreate(&e));
  float acc[3] = {0, 0, 0};
  for (int r = 0; r < reps + 1; r++) {
    CCK(cudaEventRecord(ev[0], w->s));
    w->transform(ci->definition, ev[1]);
    CCK(cudaEventRecord(ev[2], w->s));
    w->measure(ci->dir);
    CCK(cudaEventRecord(ev[3], w->s));
    CCK(cudaEventSynchronize(ev[3]));
    if (r == 0) continue;  // warm-up
    for (int k = 0; k < 3; k++) {
      float t;
      CCK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  for (int k = 0; k < 3; k++) ms[k] = acc[k] / reps;
  CCK(cudaGetLastError());
  return 0;
}

void gfix_cuts_release(void) {
  std::lock_guard<std::mutex> lk(g_work_mu);
  g_work.clear();
}

}  // extern "C"
