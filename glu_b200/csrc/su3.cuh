// SU(3) algebra for the gauge-fixing kernels, templated on the working
// precision R (double or float).  Matrices are 9 complex numbers in
// row-major order, the layout of GLU's lat[i].O[mu].
//
// The operations reproduce the reference's SSE code paths, which are what a
// default x86 build of GLU executes:
//   gram_reunit        column Gram-Schmidt, column 2 = conj(col0 x col1)
//                      (src/Matrix_Ops/gramschmidt_SSE.c:37-98)
//   set_gauge_matrix   g = reunit(1 + alpha A) from the packed fields,
//                      only columns 0 and 1 filled (src/Gfix/CG.c:72-97)
//   gtransform         b <- a b c^dag, columns 0,1 explicit, column 2 by
//                      conj cross product (src/Gfix/gtrans.c:31-141)
//   re_tr_abc_dag      Re tr(a b c^dag), row 2 of ab by cross product
//                      (src/Matrix_Ops/trace_abc_SSE.c:34-114)
//   multab             a <- b c, row 2 by cross product
//                      (src/Matrix_Ops/MMUL/MMUL_SUNC_SSE.c:30-76)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gfix {

template <typename R>
struct alignas(2 * sizeof(R)) cx {
  R x, y;
};

template <typename R>
__host__ __device__ __forceinline__ cx<R> mk(R a, R b) {
  cx<R> r;
  r.x = a;
  r.y = b;
  return r;
}

// a*b in the FMA form of the reference's SSE2_MUL
template <typename R>
__device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
  return mk<R>(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
// a*conj(b)
template <typename R>
__device__ __forceinline__ cx<R> cmulc(cx<R> a, cx<R> b) {
  return mk<R>(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -(a.x * b.y)));
}
// conj(a)*b
template <typename R>
__device__ __forceinline__ cx<R> ccmul(cx<R> a, cx<R> b) {
  return mk<R>(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -(a.y * b.x)));
}
template <typename R>
__device__ __forceinline__ cx<R> cadd(cx<R> a, cx<R> b) {
  return mk<R>(a.x + b.x, a.y + b.y);
}
template <typename R>
__device__ __forceinline__ cx<R> csub(cx<R> a, cx<R> b) {
  return mk<R>(a.x - b.x, a.y - b.y);
}
template <typename R>
__device__ __forceinline__ cx<R> conjg(cx<R> a) {
  return mk<R>(a.x, -a.y);
}
template <typename R>
__device__ __forceinline__ cx<R> cscale(cx<R> a, R s) {
  return mk<R>(a.x * s, a.y * s);
}

// column Gram-Schmidt of columns 0 (u0,u3,u6) and 1 (u1,u4,u7); column 2
// from their conjugate cross product.  The normalisations use rsqrt (within
// an ulp of GLU's 1/sqrt, far cheaper than a division and a square root).
template <typename R>
__device__ __forceinline__ void gram_reunit(cx<R> *u) {
  R n = (u[0].x * u[0].x + u[3].x * u[3].x + u[6].x * u[6].x) +
        (u[0].y * u[0].y + u[3].y * u[3].y + u[6].y * u[6].y);
  R s = rsqrt(n);
  u[0] = cscale(u[0], s);
  u[3] = cscale(u[3], s);
  u[6] = cscale(u[6], s);
  cx<R> p = cadd(cadd(cmulc(u[1], u[0]), cmulc(u[4], u[3])), cmulc(u[7], u[6]));
  u[1] = csub(u[1], cmul(p, u[0]));
  u[4] = csub(u[4], cmul(p, u[3]));
  u[7] = csub(u[7], cmul(p, u[6]));
  n = (u[1].x * u[1].x + u[4].x * u[4].x + u[7].x * u[7].x) +
      (u[1].y * u[1].y + u[4].y * u[4].y + u[7].y * u[7].y);
  s = rsqrt(n);
  u[1] = cscale(u[1], s);
  u[4] = cscale(u[4], s);
  u[7] = cscale(u[7], s);
  u[2] = conjg(csub(cmul(u[3], u[7]), cmul(u[4], u[6])));
  u[5] = conjg(csub(cmul(u[1], u[6]), cmul(u[0], u[7])));
  u[8] = conjg(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
}

// g = reunit(1 + alpha A) with A from the packed su(3) fields f0..f3
// (GLU's SU(3) packing: f0 = -D1 + i D0, f1, f2, f3 the off-diagonals)
template <typename R>
__device__ __forceinline__ void set_gauge(cx<R> *g, cx<R> f0, cx<R> f1,
                                          cx<R> f2, cx<R> f3, R alpha) {
  g[0] = mk<R>(R(1), alpha * f0.y);
  g[1] = cscale(f1, alpha);
  g[3] = mk<R>(-g[1].x, g[1].y);
  g[4] = mk<R>(R(1), -alpha * f0.x);
  g[6] = mk<R>(-alpha * f2.x, alpha * f2.y);
  g[7] = mk<R>(-alpha * f3.x, alpha * f3.y);
  gram_reunit(g);
}

// the third column of a matrix whose first two columns are set: the
// conjugate cross product of the first two, the completion of gtransform
// (src/Gfix/gtrans.c:107-121) and of gram_reunit
template <typename R>
__device__ __forceinline__ void complete_col2(cx<R> *u) {
  u[2] = conjg(csub(cmul(u[3], u[7]), cmul(u[4], u[6])));
  u[5] = conjg(csub(cmul(u[1], u[6]), cmul(u[0], u[7])));
  u[8] = conjg(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
}

// b <- a b c^dag
template <typename R>
__device__ __forceinline__ void gtransform(const cx<R> *a, cx<R> *b,
                                           const cx<R> *c) {
  // bc[r][k] = sum_j b[r][j] conj(c[k][j]), k = 0, 1
  cx<R> bc[6];
#pragma unroll
  for (int r = 0; r < 3; r++) {
#pragma unroll
    for (int k = 0; k < 2; k++) {
      bc[r * 2 + k] = cadd(cadd(cmulc(b[r * 3 + 0], c[k * 3 + 0]),
                                cmulc(b[r * 3 + 1], c[k * 3 + 1])),
                           cmulc(b[r * 3 + 2], c[k * 3 + 2]));
    }
  }
#pragma unroll
  for (int r = 0; r < 3; r++) {
#pragma unroll
    for (int k = 0; k < 2; k++) {
      b[r * 3 + k] = cadd(cadd(cmul(a[r * 3 + 0], bc[0 * 2 + k]),
                               cmul(a[r * 3 + 1], bc[1 * 2 + k])),
                          cmul(a[r * 3 + 2], bc[2 * 2 + k]));
    }
  }
  complete_col2(b);
}

// Re tr(a b c^dag), row 2 of (a b) completed by the cross product
template <typename R>
__device__ __forceinline__ R re_tr_abc_dag(const cx<R> *a, const cx<R> *b,
                                           const cx<R> *c) {
  cx<R> ab[9];
#pragma unroll
  for (int r = 0; r < 2; r++) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      ab[r * 3 + k] = cadd(cadd(cmul(a[r * 3 + 0], b[k]),
                                cmul(a[r * 3 + 1], b[3 + k])),
                           cmul(a[r * 3 + 2], b[6 + k]));
    }
  }
  ab[6] = conjg(csub(cmul(ab[1], ab[5]), cmul(ab[2], ab[4])));
  ab[7] = conjg(csub(cmul(ab[2], ab[3]), cmul(ab[0], ab[5])));
  ab[8] = conjg(csub(cmul(ab[0], ab[4]), cmul(ab[1], ab[3])));
  R sr = R(0), si = R(0);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    sr += (ab[r * 3 + 2].x * c[r * 3 + 2].x + ab[r * 3 + 1].x * c[r * 3 + 1].x) +
          ab[r * 3 + 0].x * c[r * 3 + 0].x;
    si += (ab[r * 3 + 2].y * c[r * 3 + 2].y + ab[r * 3 + 1].y * c[r * 3 + 1].y) +
          ab[r * 3 + 0].y * c[r * 3 + 0].y;
  }
  return sr + si;
}

// a <- b c, row 2 by conj cross product of rows 0 and 1
template <typename R>
__device__ __forceinline__ void multab(cx<R> *a, const cx<R> *b,
                                       const cx<R> *c) {
#pragma unroll
  for (int r = 0; r < 2; r++) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      a[r * 3 + k] = cadd(cmul(b[r * 3 + 0], c[k]),
                          cadd(cmul(b[r * 3 + 1], c[3 + k]),
                               cmul(b[r * 3 + 2], c[6 + k])));
    }
  }
  a[6] = conjg(csub(cmul(a[1], a[5]), cmul(a[2], a[4])));
  a[7] = conjg(csub(cmul(a[2], a[3]), cmul(a[0], a[5])));
  a[8] = conjg(csub(cmul(a[0], a[4]), cmul(a[1], a[3])));
}

// short Hermitian projection of U (src/Matrix_Ops/exactQ.c:400-428):
// q0, q3 real diagonals; q1, q2, q4 the upper off-diagonals
template <typename R>
__device__ __forceinline__ void herm_short(const cx<R> *U, R &q0, cx<R> &q1,
                                           cx<R> &q2, R &q3, cx<R> &q4) {
  const R i0 = U[0].y, i4 = U[4].y, i8 = U[8].y;
  q0 = (R(2) * i0 - i4 - i8) / R(3);
  q3 = (R(2) * i4 - i0 - i8) / R(3);
  // i/2 (conj(U3) - U1) = 0.5 (U3.y + U1.y) + i 0.5 (U3.x - U1.x)
  q1 = mk<R>(R(0.5) * (U[3].y + U[1].y), R(0.5) * (U[3].x - U[1].x));
  q2 = mk<R>(R(0.5) * (U[6].y + U[2].y), R(0.5) * (U[6].x - U[2].x));
  q4 = mk<R>(R(0.5) * (U[7].y + U[5].y), R(0.5) * (U[7].x - U[5].x));
}

template <typename R>
__device__ __forceinline__ void set_identity(cx<R> *u) {
#pragma unroll
  for (int k = 0; k < 9; k++) u[k] = mk<R>(R(0), R(0));
  u[0] = u[4] = u[8] = mk<R>(R(1), R(0));
}

}  // namespace gfix
