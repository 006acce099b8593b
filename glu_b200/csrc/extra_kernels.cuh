// Auxiliary kernels: observables, reunitarisation, precision switch.
#pragma once

#include "coulomb.cuh"
#include "kernels.cuh"
#include "su3_log.cuh"

namespace gfix {

// average plaquette partials: Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag
// U_nu(x)^dag) summed over mu > nu (src/Field/plaqs_links.c:243-265)
template <typename R, typename F = R>
__global__ void __launch_bounds__(kSiteThreads) k_plaquette(Ctx<R, F> c) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (s < c.V) {
    int x[4], sd[4];
    coords(s, c.L, x);
    strides(c, sd);
    cx<R> a[9], b[9], cc[9], d[9];
    double p = 0.0;
    for (int mu = 1; mu < 4; mu++) {
      const int t = fwd_site(s, mu, x, c.L, sd);
      load_link(c.U, c.V, mu, s, a);
      for (int nu = 0; nu < mu; nu++) {
        const int u = fwd_site(s, nu, x, c.L, sd);
        load_link(c.U, c.V, nu, t, b);
        load_link(c.U, c.V, mu, u, cc);
        load_link(c.U, c.V, nu, s, d);
        // ab = a b ; dc = d cc ; Re tr(ab (dc)^dag)
        double tr = 0.0;
        for (int r = 0; r < 3; r++)
          for (int k = 0; k < 3; k++) {
            cx<R> ab = mk<R>(R(0), R(0)), dc = mk<R>(R(0), R(0));
            for (int j = 0; j < 3; j++) {
              ab = cadd(ab, cmul(a[r * 3 + j], b[j * 3 + k]));
              dc = cadd(dc, cmul(d[r * 3 + j], cc[j * 3 + k]));
            }
            tr += (double)ab.x * dc.x + (double)ab.y * dc.y;
          }
        p += tr;
      }
    }
    v[0] = p;
  }
  block_sum_store<1>(v, c.part + blockIdx.x);
}

// latt_reunitU (src/Geometry/random_config.c:42-57) of the links (stored
// as their first two columns: the Gram-Schmidt needs no third)
template <typename R>
__global__ void k_reunit_links(cx<R> *U, int V) {
  const size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (l >= 4 * (size_t)V) return;
  const int mu = (int)(l / V), s = (int)(l % V);
  cx<R> u[9];
  load_link(U, V, mu, s, u);
  gram_reunit(u);
  store_link(U, V, mu, s, u);
}

// the same for n full matrices G[9][n] (gauge transforms)
template <typename R>
__global__ void k_reunit_mats(cx<R> *G, size_t n) {
  const size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  cx<R> u[9];
  cx<R> *p = G + s;
#pragma unroll
  for (int e = 0; e < 9; e++) u[e] = p[(size_t)e * n];
  gram_reunit(u);
#pragma unroll
  for (int e = 0; e < 9; e++) p[(size_t)e * n] = u[e];
}

// Link diagnostics of GLU's output (src/Field/plaqs_links.c:399-446,
// src/Gfix/gftests.c:35-129), per block of sites of one time slice t
// (grid (blocks per slice, Lt)): Re tr of the spatial and of the temporal
// links, the largest Re tr of any link, and the sum over the slice of the
// Hermitian projection of the temporal links (entries 00, 01, 02, 11, 12 of
// Hermitian_proj, exactQ.c:358-371: 8 reals), and the same 8 reals of their
// logarithm (exact_log_slow, exactQ.c:157-240).  Partials: 19 per block.
constexpr int kDiagThreads = 128;
constexpr int kDiagVals = 19;

template <typename R, typename F = R>
__global__ void __launch_bounds__(kDiagThreads) k_link_diag(Ctx<R, F> c, int lcu,
                                                             int nbs) {
  const int t = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[kDiagVals];
#pragma unroll
  for (int k = 0; k < kDiagVals; k++) v[k] = 0.0;
  v[2] = -1e300;
  if (i < lcu) {
    const int s = t * lcu + i;
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
      cx<R> u[9];
      load_link(c.U, c.V, mu, s, u);
      const double tr = (double)u[0].x + (double)u[4].x + (double)u[8].x;
      if (mu < 3)
        v[0] += tr;
      else
        v[1] += tr;
      v[2] = fmax(v[2], tr);
      if (mu == 3) {
        const double i0 = u[0].y, i4 = u[4].y, i8 = u[8].y;
        v[3] += (2 * i0 - i4 - i8) / 3.;
        // -i (a - conj(b)) / 2 = ((a.y + b.y) / 2, -(a.x - b.x) / 2)
        v[4] += 0.5 * ((double)u[1].y + (double)u[3].y);
        v[5] += -0.5 * ((double)u[1].x - (double)u[3].x);
        v[6] += 0.5 * ((double)u[2].y + (double)u[6].y);
        v[7] += -0.5 * ((double)u[2].x - (double)u[6].x);
        v[8] += (2 * i4 - i0 - i8) / 3.;
        v[9] += 0.5 * ((double)u[5].y + (double)u[7].y);
        v[10] += -0.5 * ((double)u[5].x - (double)u[7].x);
        cx<double> ud[9], q[4];
#pragma unroll
        for (int e = 0; e < 9; e++) ud[e] = mk<double>((double)u[e].x, (double)u[e].y);
        su3log::log_components(ud, q);  // (Q00 + i Q11, Q01, Q02, Q12)
        v[11] += q[0].x;
        v[12] += q[1].x;
        v[13] += q[1].y;
        v[14] += q[2].x;
        v[15] += q[2].y;
        v[16] += q[0].y;
        v[17] += q[3].x;
        v[18] += q[3].y;
      }
    }
  }
  // sums (the maximum through its own warp and block reduction)
  double m = v[2];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double smax[kDiagThreads / 32];
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
  v[2] = 0.0;
  double *out = c.part + (size_t)kDiagVals * ((size_t)t * nbs + blockIdx.x);
  block_sum_store<kDiagVals>(v, out);
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = smax[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mm = fmax(mm, smax[w]);
    out[2] = mm;
  }
}

template <typename R>
__global__ void k_identity(cx<R> *G, int V) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
#pragma unroll
  for (int e = 0; e < 9; e++)
    G[(size_t)e * V + s] = mk<R>(R(e == 0 || e == 4 || e == 8), R(0));
}

// element-wise precision conversion of n complex numbers
template <typename RS, typename RD>
__global__ void k_convert(const cx<RS> *a, cx<RD> *b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = mk<RD>((RD)a[i].x, (RD)a[i].y);
}

// U_mu(x) <- G(x) U_mu(x) G(x+mu)^dag with G widened to FP64 and
// reunitarised first; used when the FP32 phase hands its accumulated
// transform (G in RG, FP32) to the FP64 links
template <typename F, typename RG>
__global__ void __launch_bounds__(kSiteThreads)
    k_apply_gauge(Ctx<double, F> c, const cx<RG> *G) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.V) return;
  int x[4], sd[4];
  coords(s, c.L, x);
  strides(c, sd);
  const size_t V = c.V;
  cx<double> A[9], B[9], U[9];
#pragma unroll
  for (int e = 0; e < 9; e++)
    A[e] = mk<double>((double)G[(size_t)e * V + s].x, (double)G[(size_t)e * V + s].y);
  gram_reunit(A);
  for (int mu = 0; mu < 4; mu++) {
    const int y = fwd_site(s, mu, x, c.L, sd);
#pragma unroll
    for (int e = 0; e < 9; e++)
      B[e] = mk<double>((double)G[(size_t)e * V + y].x, (double)G[(size_t)e * V + y].y);
    gram_reunit(B);
    load_link(c.U, c.V, mu, s, U);
    gtransform(A, U, B);
    store_link(c.U, c.V, mu, s, U);
  }
}

// The random SU(3) gauge matrix of site s for a random restart of a Landau
// fix (GLU's random_transform, src/Geometry/random_config.c:107-120, which
// draws them from its own per-thread generator): nine complex Gaussian
// entries (Box-Muller on a SplitMix64 stream keyed by the seed, the
// attempt and the site), then the column Gram-Schmidt of gram_reunit
// (columns 0 and 1 orthonormal, column 2 their conjugate cross product).
// Reproducible for a given (seed, attempt); not GLU's stream.
__device__ __forceinline__ void random_su3(cx<double> *g, unsigned long long seed,
                                           int attempt, int s) {
  unsigned long long h =
      mix64(seed ^ mix64(((unsigned long long)attempt << 40) ^ (unsigned long long)s));
#pragma unroll
  for (int e = 0; e < 9; e++) {
    h = mix64(h);
    const double u1 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    h = mix64(h);
    const double u2 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double rad = sqrt(-2.0 * log(u1));
    g[e] = mk<double>(rad * cospi(2.0 * u2), rad * sinpi(2.0 * u2));
  }
  gram_reunit(g);
}

// U_mu(x) <- g(x) U_mu(x) g(x + mu)^dag with the random matrices of
// random_su3 (each site's drawn again by its -mu neighbours: no buffer)
template <typename F>
__global__ void __launch_bounds__(kSiteThreads)
    k_random_transform(Ctx<double, F> c, unsigned long long seed, int attempt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.V) return;
  int x[4], sd[4];
  coords(s, c.L, x);
  strides(c, sd);
  cx<double> A[9], B[9], U[9];
  random_su3(A, seed, attempt, s);
#pragma unroll 1
  for (int mu = 0; mu < 4; mu++) {
    random_su3(B, seed, attempt, fwd_site(s, mu, x, c.L, sd));
    load_link(c.U, c.V, mu, s, U);
    gtransform(A, U, B);
    store_link(c.U, c.V, mu, s, U);
  }
}

// GLU's gauge-fixing accuracy report (gf_check, src/Wrappers/OBS_wrap.c:
// 93-126): per site the lattice derivative sum_mu [A_mu(x - mu) - A_mu(x)]
// of the Hermitian fields A of the links, by the linear definition
// (Hermitian_proj_short, as theta_test_lin, src/Gfix/gftests.c:214-250)
// and the logarithmic one (exact_log_slow_short, as theta_test_log,
// gftests.c:253-290, through log_deriv, src/Gfix/log_derivs.c:29-50), over
// the four directions (Landau) and the three spatial ones (Coulomb); the
// local value is trace_deriv (src/Gfix/lin_derivs.c:29-52).  Per block:
// the sums of the four local values and their maxima, kGfcVals doubles.
constexpr int kGfcVals = 8;

__device__ __forceinline__ double gfc_trace_deriv(const double *r) {
  // r = {Re s0, Re s3, s1, s2, s4 (re, im)}
  return 4.0 * (r[0] * r[0] + r[1] * r[1] + r[0] * r[1] + r[2] * r[2] + r[3] * r[3] +
                r[4] * r[4] + r[5] * r[5] + r[6] * r[6] + r[7] * r[7]);
}

// the eight reals of a short Hermitian field: linear definition
__device__ __forceinline__ void gfc_lin(const cx<double> *u, double *a) {
  double q0, q3;
  cx<double> q1, q2, q4;
  herm_short(u, q0, q1, q2, q3, q4);
  a[0] = q0;
  a[1] = q3;
  a[2] = q1.x;
  a[3] = q1.y;
  a[4] = q2.x;
  a[5] = q2.y;
  a[6] = q4.x;
  a[7] = q4.y;
}

// logarithmic definition: (Re Q00, Re Q11, Q01, Q02, Q12)
__device__ __forceinline__ void gfc_log(const cx<double> *u, double *a) {
  cx<double> q[4];
  su3log::log_components(u, q);
  a[0] = q[0].x;
  a[1] = q[0].y;
  a[2] = q[1].x;
  a[3] = q[1].y;
  a[4] = q[2].x;
  a[5] = q[2].y;
  a[6] = q[3].x;
  a[7] = q[3].y;
}

template <typename F>
__global__ void __launch_bounds__(kSiteThreads) k_gf_check(Ctx<double, F> c) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  // {lin 4D, log 4D, lin 3D, log 3D}
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (s < c.V) {
    int x[4], sd[4];
    coords(s, c.L, x);
    strides(c, sd);
    double sl[8] = {0, 0, 0, 0, 0, 0, 0, 0}, sg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
      cx<double> u[9], b[9];
      load_link(c.U, c.V, mu, s, u);
      load_link(c.U, c.V, mu, bck_site(s, mu, x, c.L, sd), b);
      double a[8], ab[8];
      gfc_lin(u, a);
      gfc_lin(b, ab);
#pragma unroll
      for (int k = 0; k < 8; k++) sl[k] += ab[k] - a[k];
      gfc_log(u, a);
      gfc_log(b, ab);
#pragma unroll
      for (int k = 0; k < 8; k++) sg[k] += ab[k] - a[k];
      if (mu == 2) {
        v[2] = gfc_trace_deriv(sl);
        v[3] = gfc_trace_deriv(sg);
      }
    }
    v[0] = gfc_trace_deriv(sl);
    v[1] = gfc_trace_deriv(sg);
  }
  double m[4] = {v[0], v[1], v[2], v[3]};
  double *out = c.part + (size_t)kGfcVals * blockIdx.x;
  block_sum_store<4>(v, out);
  __shared__ double smax[4][kSiteThreads / 32];
#pragma unroll
  for (int k = 0; k < 4; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m[k] = fmax(m[k], __shfl_down_sync(0xffffffffu, m[k], o));
    if ((threadIdx.x & 31) == 0) smax[k][threadIdx.x >> 5] = m[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 4; k++) {
      double mm = smax[k][0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) mm = fmax(mm, smax[k][w]);
      out[4 + k] = mm;
    }
  }
}

}  // namespace gfix
