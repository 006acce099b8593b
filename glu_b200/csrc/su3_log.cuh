// The SU(3) matrix logarithm of GLU's LOGARITHMIC field definition, FP64
// device code shared by the momentum-space measurements (cuts.cu) and the
// post-fix link diagnostics (extra_kernels.cuh).
#pragma once

#include "su3.cuh"

namespace gfix {
namespace su3log {

using C2 = cx<double>;

__device__ __forceinline__ C2 cm(C2 a, C2 b) {
  return mk<double>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// The logarithmic definition (exact_log_slow, src/Matrix_Ops/exactQ.c:
// 157-240): eigenvalues of the link from its characteristic cubic
// (Eigenvalues_suNC, src/Matrix_Ops/evalues.c:317-349, and the
// near-identity form Eigenvalues_su3_stab, evalues.c:185-202), their
// phases, and Q = log(U)/i from the su(3) f-constants
// (f_hermitian_log_suNC, src/Matrix_Ops/effs.c:63-95).

__device__ __forceinline__ C2 cadd2(C2 a, C2 b) { return mk<double>(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ C2 csub2(C2 a, C2 b) { return mk<double>(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ C2 cscal(C2 a, double s) { return mk<double>(a.x * s, a.y * s); }
__device__ __forceinline__ C2 cconj(C2 a) { return mk<double>(a.x, -a.y); }
__device__ __forceinline__ C2 cdiv(C2 a, C2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return mk<double>((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// GLU's squarert keeps the real part of the root only (its result is a
// double); for an SU(3) link the argument -- minus the cubic's
// discriminant over 108 -- is real and non-negative, so this is the root
__device__ __forceinline__ double sq_root(C2 z, C2 R) {
  const double t = sqrt(hypot(z.x, z.y)) * cos(atan2(z.y, z.x) * 0.5);
  return (R.x * t < 0) ? -t : t;
}

__device__ __forceinline__ C2 cube_root(C2 z) {
  const double r = cbrt(hypot(z.x, z.y));
  const double a = atan2(z.y, z.x) / 3.;
  return mk<double>(r * cos(a), r * sin(a));
}

__device__ inline void su3_eigenvalues(const C2 *U, C2 z[3]) {
  const C2 rr3 = mk<double>(0., 1.7320508075688772);  // i sqrt(3)
  const C2 tr = cadd2(cadd2(U[0], U[4]), U[8]);
  if (1.0 - (U[0].x + U[4].x + U[8].x) / 3. < 1E-12) {
    // eigenvalues of 1 - U near the identity
    const C2 a = mk<double>(1.0 - tr.x / 3., -(tr.y / 3.));
    const C2 b = mk<double>(-a.x, a.y);
    const C2 p = cadd2(b, cm(a, mk<double>(2.0 - a.x, -a.y)));
    const C2 t1 = mk<double>(1.0 - a.x / 3., -(a.y / 3.));
    const C2 inner = csub2(csub2(mk<double>(1.0, 0.0), b), cm(cscal(a, 2.0), t1));
    const C2 q = cscal(cadd2(cm(a, inner), b), 1.5);
    const double res = sq_root(cadd2(cm(q, q), cm(cm(p, p), p)), p);
    const C2 u1 = cube_root(mk<double>(res - q.x, -q.y));
    const C2 u2 = (u1.x != 0.0) ? cdiv(mk<double>(-p.x, -p.y), u1) : mk<double>(0., 0.);
    const C2 plus = cadd2(u1, u2);
    const C2 minus = cm(rr3, csub2(u1, u2));
    z[0] = csub2(cadd2(mk<double>(1.0, 0.0), plus), a);
    z[1] = csub2(cadd2(mk<double>(1.0, 0.0), cscal(csub2(minus, plus), 0.5)), a);
    z[2] = csub2(z[1], minus);
    return;
  }
  const C2 a = mk<double>(-tr.x / 3., -tr.y / 3.);
  const C2 ca = cconj(a);
  const C2 Q = cadd2(cm(a, a), ca);
  const C2 R = csub2(cm(a, cadd2(Q, cscal(ca, 0.5))), mk<double>(0.5, 0.0));
  const C2 temp = csub2(cm(R, R), cm(cm(Q, Q), Q));
  const double res = sq_root(temp, R);
  const C2 A = cscal(cube_root(mk<double>(R.x + res, R.y)), -1.0);
  const C2 B = (A.x != 0.0 || A.y != 0.0) ? cdiv(Q, A) : mk<double>(0., 0.);
  const C2 plus = cadd2(A, B);
  const C2 minus = cm(rr3, csub2(A, B));
  z[0] = csub2(plus, a);
  z[1] = csub2(cscal(csub2(minus, plus), 0.5), a);
  z[2] = csub2(z[1], minus);
}

// the four packed components of exact_log_slow(U); zero where GLU's
// routine returns without writing (all three phases equal, i.e. U = 1)
__device__ inline void log_components(const C2 *U, C2 out[4]) {
  C2 ev[3];
  su3_eigenvalues(U, ev);
  const double z0 = atan2(ev[0].y, ev[0].x), z1 = atan2(ev[1].y, ev[1].x);
  const double z2 = -(z0 - z1);
  if (z0 == z1 && z1 == z2) {
    for (int k = 0; k < 4; k++) out[k] = mk<double>(0., 0.);
    return;
  }
  const double u = 0.5 * z0, w = z1 + u;
  const double cw = cos(w), cu = cos(u), su = sin(u);
  const C2 one1 = mk<double>(cu, -su);
  const C2 two1 = cm(cconj(one1), cconj(one1));
  const double uu = u * u, ww = w * w;
  const double denom = 1.0 / (9. * uu - ww);
  const double E0 = fabs(w) < 1E-13 ? 1 - ww / 6. * (1 - ww / 20. * (1 - ww / 42.)) : sin(w) / w;
  C2 f0 = cadd2(cscal(two1, uu - ww),
                cm(one1, mk<double>(8. * uu * cw, 2. * u * (3. * uu + ww) * E0)));
  C2 f1 = csub2(cscal(two1, 2 * u), cm(one1, mk<double>(2. * u * cw, -((3. * uu - ww) * E0))));
  C2 f2 = csub2(two1, cm(one1, mk<double>(cw, 3. * u * E0)));
  f0 = cscal(f0, denom);
  f1 = cscal(f1, denom);
  f2 = cscal(f2, denom);
  const C2 con = cconj(f2);
  const double mod = 1.0 / (f1.y * f2.x - f1.x * f2.y);
  const double imf = (f0.y * f2.x - f0.x * f2.y) * mod;
  const C2 trce = mk<double>(0., -mod / 2.);
  auto entry = [&](C2 uab, C2 uba) { return cm(trce, csub2(cm(con, uab), cm(f2, cconj(uba)))); };
  const C2 q0 = entry(U[0], U[0]), q4 = entry(U[4], U[4]);
  out[0] = mk<double>(q0.x - imf, q4.x - imf);
  out[1] = entry(U[1], U[3]);
  out[2] = entry(U[2], U[6]);
  out[3] = entry(U[5], U[7]);
}

}  // namespace su3log
}  // namespace gfix
