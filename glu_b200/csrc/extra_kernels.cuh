// Auxiliary kernels: observables, reunitarisation, precision switch.
#pragma once

#include "kernels.cuh"

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

}  // namespace gfix
