// Auxiliary kernels: observables, reunitarisation, precision switch.
#pragma once

#include "coulomb.cuh"
#include "kernels.cuh"
#include "su3_log.cuh"

namespace gfix {

// average plaquette partials: Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag
// U_nu(x)^dag) summed over mu > nu (src/Field/plaqs_links.c:243-265)
template <typename R>
__global__ void __launch_bounds__(kSiteThreads) k_plaquette(Ctx<R> c) {
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

template <typename R>
__global__ void k_reunit_links(cx<R> *U, size_t nlinks, size_t V) {
  const size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const size_t mu = l / V, s = l % V;
  cx<R> u[9];
  cx<R> *p = U + mu * 9 * V + s;
#pragma unroll
  for (int e = 0; e < 9; e++) u[e] = p[(size_t)e * V];
  gram_reunit(u);
#pragma unroll
  for (int e = 0; e < 9; e++) p[(size_t)e * V] = u[e];
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

template <typename R>
__global__ void __launch_bounds__(kDiagThreads) k_link_diag(Ctx<R> c, int lcu,
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

// U_mu(x) <- G(x) U_mu(x) G(x+mu)^dag with G reunitarised first (FP64);
// used when the FP32 phase hands its accumulated transform to FP64
__global__ void __launch_bounds__(kSiteThreads)
    k_apply_gauge(Ctx<double> c, const cx<double> *G) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.V) return;
  int x[4], sd[4];
  coords(s, c.L, x);
  strides(c, sd);
  const size_t V = c.V;
  cx<double> A[9], B[9], U[9];
#pragma unroll
  for (int e = 0; e < 9; e++) A[e] = G[(size_t)e * V + s];
  gram_reunit(A);
  for (int mu = 0; mu < 4; mu++) {
    const int y = fwd_site(s, mu, x, c.L, sd);
#pragma unroll
    for (int e = 0; e < 9; e++) B[e] = G[(size_t)e * V + y];
    gram_reunit(B);
    load_link(c.U, c.V, mu, s, U);
    gtransform(A, U, B);
    store_link(c.U, c.V, mu, s, U);
  }
}

// Random SU(3) gauge matrices G[9][V] for a random restart of a Landau fix
// (GLU's random_transform, src/Geometry/random_config.c:107-120, which
// draws them from its own per-thread generator): per site nine complex
// Gaussian entries (Box-Muller on a SplitMix64 stream keyed by the seed,
// the attempt and the site), then the column Gram-Schmidt of gram_reunit
// (columns 0 and 1 orthonormal, column 2 their conjugate cross product).
// Reproducible for a given (seed, attempt); not GLU's stream.
__global__ void k_random_gauge(cx<double> *G, int V, unsigned long long seed,
                               int attempt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  unsigned long long h =
      mix64(seed ^ mix64(((unsigned long long)attempt << 40) ^ (unsigned long long)s));
  cx<double> g[9];
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
#pragma unroll
  for (int e = 0; e < 9; e++) G[(size_t)e * V + s] = g[e];
}

}  // namespace gfix
