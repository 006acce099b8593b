/*
 * CPU oracle for GLU's Fourier-accelerated gauge fixing: our own plain-C
 * restatement, single threaded, FP64.  TEST INFRASTRUCTURE ONLY (see
 * gfix_oracle.h): nothing in glu_b200/ uses it.
 *
 * It follows the reference's serial (one OpenMP thread) evaluation order,
 * including the quirks that change results: the packed SU(3) inner
 * products, Kahan sums where GLU uses them, the reduction-array contents
 * that carry into a continuation run, the line-search clipping and the
 * CG_TOL switches.  Column 2 of every product is completed by a conjugate
 * cross product as GLU's SSE code paths do.
 */
#include "gfix_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

typedef double complex cpx;

#define NC 3
#define ND 4
#define NCNC 9
#define NF 4                 /* TRUE_HERM for SU(3) */
#define LINE_NSTEPS 3        /* src/Headers/GLU_definitions.h:461 */
#define CG_TOL 5E-11         /* src/Headers/GLU_definitions.h:451-455 */
#define PREC_TOL (NC * 1.0E-14)
#define TWOPI_GLU (6.283185307179586) /* GLU_definitions.h:139 */
#define VAL49 0.4444444444444444      /* lin_derivs.c:72 */

/* ------------------------------------------------------------------ */
/* geometry: site i = x + Lx (y + Ly (z + Lz t)), periodic            */

typedef struct {
  size_t dims[ND];
  size_t V, Lcu;
  size_t *fwd, *bck; /* [V][ND] */
} geom_t;

static int geom_init(geom_t *g, const size_t dims[ND]) {
  g->V = 1;
  for (int mu = 0; mu < ND; mu++) {
    g->dims[mu] = dims[mu];
    g->V *= dims[mu];
  }
  g->Lcu = dims[0] * dims[1] * dims[2];
  g->fwd = (size_t *)malloc(sizeof(size_t) * g->V * ND);
  g->bck = (size_t *)malloc(sizeof(size_t) * g->V * ND);
  if (!g->fwd || !g->bck) return -1;
  for (size_t i = 0; i < g->V; i++) {
    size_t x[ND], r = i;
    for (int mu = 0; mu < ND; mu++) {
      x[mu] = r % dims[mu];
      r /= dims[mu];
    }
    for (int mu = 0; mu < ND; mu++) {
      size_t xf[ND], xb[ND];
      memcpy(xf, x, sizeof(x));
      memcpy(xb, x, sizeof(x));
      xf[mu] = (x[mu] + 1) % dims[mu];
      xb[mu] = (x[mu] + dims[mu] - 1) % dims[mu];
      size_t jf = 0, jb = 0;
      for (int nu = ND - 1; nu >= 0; nu--) {
        jf = jf * dims[nu] + xf[nu];
        jb = jb * dims[nu] + xb[nu];
      }
      g->fwd[i * ND + mu] = jf;
      g->bck[i * ND + mu] = jb;
    }
  }
  return 0;
}

static void geom_free(geom_t *g) {
  free(g->fwd);
  free(g->bck);
}

/* ------------------------------------------------------------------ */
/* SU(3) helpers                                                      */

static inline cpx cm(cpx a, cpx b) { /* a*b, as the SSE2_MUL FMA form */
  const double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
  return fma(ar, br, -(ai * bi)) + I * fma(ar, bi, ai * br);
}

/* column Gram-Schmidt with a conj-cross-product third column
 * (src/Matrix_Ops/gramschmidt_SSE.c:37-98; columns are u[0,3,6], u[1,4,7]) */
static void gram_reunit_c(cpx *u) {
  double n0r = creal(u[0]) * creal(u[0]) + creal(u[3]) * creal(u[3]) +
               creal(u[6]) * creal(u[6]);
  double n0i = cimag(u[0]) * cimag(u[0]) + cimag(u[3]) * cimag(u[3]) +
               cimag(u[6]) * cimag(u[6]);
  double s = 1.0 / sqrt(n0r + n0i);
  u[0] *= s; u[3] *= s; u[6] *= s;
  /* <col0, col1> = sum u1 conj(u0) */
  cpx p = u[1] * conj(u[0]) + u[4] * conj(u[3]) + u[7] * conj(u[6]);
  u[1] -= cm(p, u[0]);
  u[4] -= cm(p, u[3]);
  u[7] -= cm(p, u[6]);
  double n1r = creal(u[1]) * creal(u[1]) + creal(u[4]) * creal(u[4]) +
               creal(u[7]) * creal(u[7]);
  double n1i = cimag(u[1]) * cimag(u[1]) + cimag(u[4]) * cimag(u[4]) +
               cimag(u[7]) * cimag(u[7]);
  s = 1.0 / sqrt(n1r + n1i);
  u[1] *= s; u[4] *= s; u[7] *= s;
  u[2] = conj(cm(u[3], u[7]) - cm(u[4], u[6]));
  u[5] = conj(cm(u[1], u[6]) - cm(u[0], u[7]));
  u[8] = conj(cm(u[0], u[4]) - cm(u[1], u[3]));
}

/* g = reunit(1 + alpha A(x)) from the packed fields, only columns 0 and 1
 * are filled before reunitarisation (src/Gfix/CG.c:72-97) */
static void set_gauge_matrix_c(cpx *gx, cpx *const *in, double alpha,
                               size_t i) {
  gx[0] = 1.0 + I * alpha * cimag(in[0][i]);
  gx[1] = alpha * in[1][i];
  gx[3] = -conj(gx[1]);
  gx[4] = 1.0 - I * alpha * creal(in[0][i]);
  gx[6] = -alpha * conj(in[2][i]);
  gx[7] = -alpha * conj(in[3][i]);
  gx[2] = gx[5] = gx[8] = 0.0;
  gram_reunit_c(gx);
}

/* b <- a b c^dag, columns 0 and 1 explicit, column 2 by conj cross
 * product (src/Gfix/gtrans.c:31-141) */
static void gtransform_local_c(const cpx *a, cpx *b, const cpx *c) {
  cpx bc[6]; /* (b c^dag) columns 0,1: bc[r*2+k] = sum_j b[r][j] conj(c[k][j]) */
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 2; k++) {
      cpx s = 0.0;
      for (int j = 0; j < 3; j++) s += b[r * 3 + j] * conj(c[k * 3 + j]);
      bc[r * 2 + k] = s;
    }
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 2; k++) {
      cpx s = 0.0;
      for (int j = 0; j < 3; j++) s += a[r * 3 + j] * bc[j * 2 + k];
      b[r * 3 + k] = s;
    }
  b[2] = conj(cm(b[3], b[7]) - cm(b[4], b[6]));
  b[5] = conj(cm(b[1], b[6]) - cm(b[0], b[7]));
  b[8] = conj(cm(b[0], b[4]) - cm(b[1], b[3]));
}

/* a <- b c with row 2 completed by conj cross product
 * (src/Matrix_Ops/MMUL/MMUL_SUNC_SSE.c:30-76) */
static void multab_suNC_c(cpx *a, const cpx *b, const cpx *c) {
  for (int r = 0; r < 2; r++)
    for (int k = 0; k < 3; k++)
      a[r * 3 + k] = cm(b[r * 3 + 0], c[k]) +
                     (cm(b[r * 3 + 1], c[3 + k]) + cm(b[r * 3 + 2], c[6 + k]));
  a[6] = conj(cm(a[1], a[5]) - cm(a[2], a[4]));
  a[7] = conj(cm(a[2], a[3]) - cm(a[0], a[5]));
  a[8] = conj(cm(a[0], a[4]) - cm(a[1], a[3]));
}

/* Re tr(a b c^dag) with row 2 of (a b) from the cross product of its rows
 * 0 and 1 (src/Matrix_Ops/trace_abc_SSE.c:34-114) */
static double re_trace_abc_dag_c(const cpx *a, const cpx *b, const cpx *c) {
  cpx ab[9];
  for (int r = 0; r < 2; r++)
    for (int k = 0; k < 3; k++)
      ab[r * 3 + k] =
          (cm(a[r * 3 + 0], b[k]) + cm(a[r * 3 + 1], b[3 + k])) +
          cm(a[r * 3 + 2], b[6 + k]);
  ab[6] = conj(cm(ab[1], ab[5]) - cm(ab[2], ab[4]));
  ab[7] = conj(cm(ab[2], ab[3]) - cm(ab[0], ab[5]));
  ab[8] = conj(cm(ab[0], ab[4]) - cm(ab[1], ab[3]));
  double sr = 0.0, si = 0.0;
  for (int r = 0; r < 3; r++) {
    double er = 0.0, ei = 0.0;
    for (int k = 2; k >= 0; k--) {
      er += creal(ab[r * 3 + k]) * creal(c[r * 3 + k]);
      ei += cimag(ab[r * 3 + k]) * cimag(c[r * 3 + k]);
    }
    sr += er;
    si += ei;
  }
  return sr + si;
}

/* short Hermitian projection (src/Matrix_Ops/exactQ.c:400-428) */
static void hermitian_proj_short_c(cpx *Q, const cpx *U) {
  const double i0 = cimag(U[0]), i4 = cimag(U[4]), i8 = cimag(U[8]);
  Q[0] = (2. * i0 - i4 - i8) / 3.;
  Q[1] = I * 0.5 * (conj(U[3]) - U[1]);
  Q[2] = I * 0.5 * (conj(U[6]) - U[2]);
  Q[3] = (2. * i4 - i0 - i8) / 3.;
  Q[4] = I * 0.5 * (conj(U[7]) - U[5]);
}

static void identity_c(cpx *u) {
  for (int k = 0; k < 9; k++) u[k] = 0.0;
  u[0] = u[4] = u[8] = 1.0;
}

static inline void kahan_add(double *sum, double *c, double v) {
  const double y = v - *c;
  const double t = *sum + y;
  *c = (t - *sum) - y;
  *sum = t;
}

/* ------------------------------------------------------------------ */
/* Landau derivative (src/Gfix/lin_derivs.c:74-193, FACG.c:38-73)      */

static double fa_deriv(cpx *const *in, const cpx *U, const geom_t *g) {
  double red = 0.0;
  for (size_t i = 0; i < g->V; i++) {
    double R0 = 0., R1 = 0., I1 = 0., R2 = 0., I2 = 0., R3 = 0., R4 = 0.,
           I4 = 0.;
    for (int mu = 0; mu < ND; mu++) {
      const double *q = (const double *)(U + (i * ND + mu) * NCNC);
      const double *s =
          (const double *)(U + (g->bck[i * ND + mu] * ND + mu) * NCNC);
      R0 += 2 * s[1] - s[9] - s[17];
      R0 += -2 * q[1] + q[9] + q[17];
      R1 += s[2] - s[6] - q[2] + q[6];
      I1 += s[3] + s[7] - q[3] - q[7];
      R2 += s[4] - s[12] - q[4] + q[12];
      I2 += s[5] + s[13] - q[5] - q[13];
      R3 += 2 * s[9] - s[1] - s[17];
      R3 += -2 * q[9] + q[1] + q[17];
      R4 += s[10] - s[14] - q[10] + q[14];
      I4 += s[11] + s[15] - q[11] - q[15];
    }
    const double sum0 = R0 / 3., sum3 = R3 / 3.;
    in[0][i] = -sum3 + I * sum0;
    in[1][i] = 0.5 * R1 + I * (0.5 * I1);
    in[2][i] = 0.5 * R2 + I * (0.5 * I2);
    in[3][i] = 0.5 * R4 + I * (0.5 * I4);
    red += VAL49 * (R0 * R0 + R3 * (R3 + R0)) +
           (R1 * R1 + I1 * I1 + R2 * R2 + I2 * I2 + R4 * R4 + I4 * I4);
  }
  return red;
}

/* ------------------------------------------------------------------ */
/* p^2 table and the accelerated gradient                              */

/* psq[i] = MAX / p^2(i), p^2 = 2 (D - sum cos(2 pi n_mu / L_mu)), p=0 -> 1
 * (src/Geometry/geometry.c:169-186, src/Gfix/Landau.c:277-284,
 * src/Gfix/Coulomb.c:53-59) */
void orc_psq(double *psq, const size_t dims[4], int ndim) {
  size_t vol = 1;
  for (int mu = 0; mu < ndim; mu++) vol *= dims[mu];
  const double maxp = 4. * (double)ndim / (double)vol;
  for (size_t i = 0; i < vol; i++) {
    size_t r = i;
    double kcos = 0.;
    for (int mu = 0; mu < ndim; mu++) {
      const int n = (int)(r % dims[mu]);
      r /= dims[mu];
      kcos += cos(n * (TWOPI_GLU / (double)dims[mu]));
    }
    const double p2 = (kcos == (double)ndim) ? 1.0 : 2.0 * ((double)ndim - kcos);
    psq[i] = maxp / p2;
  }
}

typedef struct {
  int ndim;
  size_t vol;
  cpx *out[NF];
  fftw_plan fwd[NF], bwd[NF];
  double *psq;
} fa_t;

static int fa_init(fa_t *f, cpx *const *in, const size_t dims[4], int ndim) {
  int n[ND];
  f->ndim = ndim;
  f->vol = 1;
  for (int mu = 0; mu < ndim; mu++) {
    n[mu] = (int)dims[ndim - 1 - mu]; /* slowest first (plan_ffts.c:113) */
    f->vol *= dims[mu];
  }
  f->psq = (double *)malloc(sizeof(double) * f->vol);
  if (!f->psq) return -1;
  orc_psq(f->psq, dims, ndim);
  for (int k = 0; k < NF; k++) {
    f->out[k] = (cpx *)fftw_malloc(sizeof(cpx) * f->vol);
    f->fwd[k] = fftw_plan_dft(ndim, n, (fftw_complex *)in[k],
                              (fftw_complex *)f->out[k], FFTW_FORWARD,
                              FFTW_ESTIMATE);
    f->bwd[k] = fftw_plan_dft(ndim, n, (fftw_complex *)f->out[k],
                              (fftw_complex *)in[k], FFTW_BACKWARD,
                              FFTW_ESTIMATE);
  }
  return 0;
}

static void fa_free(fa_t *f) {
  for (int k = 0; k < NF; k++) {
    fftw_destroy_plan(f->fwd[k]);
    fftw_destroy_plan(f->bwd[k]);
    fftw_free(f->out[k]);
  }
  free(f->psq);
}

/* FOURIER_ACCELERATE3/2 (src/Gfix/FACG.c:77-95, CFACG.c:69-88) */
static void fa_apply(fa_t *f) {
  for (int k = 0; k < NF; k++) {
    fftw_execute(f->fwd[k]);
    for (size_t i = 0; i < f->vol; i++) f->out[k][i] *= f->psq[i];
    fftw_execute(f->bwd[k]);
  }
}

/* ------------------------------------------------------------------ */
/* Landau reductions, line search, link update                         */

/* sum_PR3 (src/Gfix/FACG.c:99-145) */
static void sum_pr3(cpx *const *in, cpx *const *old, size_t V,
                    double *insum, double *conjsum) {
  for (size_t i = 0; i < V; i++) {
    double l1 = 0.0, l2 = 0.0;
    const double a = creal(in[0][i]), b = cimag(in[0][i]);
    l1 += 2.0 * (a * a + b * b + a * b);
    for (int k = 1; k < NF; k++)
      l1 += 2.0 * (creal(in[k][i]) * creal(in[k][i]) +
                   cimag(in[k][i]) * cimag(in[k][i]));
    cpx t = in[0][i] - old[0][i];
    l2 += 2.0 * (a * creal(t) + b * cimag(t));
    l2 += a * cimag(t) + b * creal(t);
    for (int k = 1; k < NF; k++) {
      t = in[k][i] - old[k][i];
      l2 += 2.0 * (creal(in[k][i]) * creal(t) + cimag(in[k][i]) * cimag(t));
    }
    *insum += l1;
    *conjsum += l2;
  }
}

/* sum_DER3 (src/Gfix/FACG.c:148-178) */
static void sum_der3(cpx *const *in, size_t V, double *red) {
  for (size_t i = 0; i < V; i++) {
    double l = 0.0;
    const double a = creal(in[0][i]), b = cimag(in[0][i]);
    l += a * a + b * b + a * b;
    for (int k = 1; k < NF; k++)
      l += creal(in[k][i]) * creal(in[k][i]) +
           cimag(in[k][i]) * cimag(in[k][i]);
    *red += 2 * l;
  }
}

double orc_approx_minimum(const double *al, const double *f) {
  const double A = f[0] / ((al[0] - al[1]) * (al[0] - al[2]));
  const double B = f[1] / ((al[1] - al[0]) * (al[1] - al[2]));
  const double C = f[2] / ((al[2] - al[0]) * (al[2] - al[1]));
  const double Sol = (al[0] * (B + C) + al[1] * (A + C) + al[2] * (A + B)) /
                     (2 * (A + B + C));
  if (Sol > al[2]) return al[2];
  if (isnan(Sol) || isinf(Sol) || Sol < al[0]) return 0.08;
  return Sol;
}

/* egauge_Landau (src/Gfix/line_search.c:60-97) */
static void egauge_landau(cpx *U, cpx *const *in, double alpha,
                          const geom_t *g) {
  for (size_t i = 0; i < g->V; i++) {
    cpx A[9], B[9];
    set_gauge_matrix_c(A, in, alpha, i);
    for (int mu = 0; mu < ND; mu++) {
      set_gauge_matrix_c(B, in, alpha, g->fwd[i * ND + mu]);
      gtransform_local_c(A, U + (i * ND + mu) * NCNC, B);
    }
  }
}

/* probe sums of line_search_Landau (src/Gfix/line_search.c:278-318), Kahan
 * accumulated onto red[0..2] */
static void landau_probes(const cpx *U, cpx *const *in, const geom_t *g,
                          double *red) {
  double c[LINE_NSTEPS] = {0., 0., 0.};
  for (size_t i = 0; i < g->V; i++) {
    cpx A1[9], A2[9], B[9];
    double v[LINE_NSTEPS] = {0., 0., 0.};
    set_gauge_matrix_c(A1, in, 0.15, i);
    set_gauge_matrix_c(A2, in, 0.30, i);
    for (int mu = 0; mu < ND; mu++) {
      const cpx *u = U + (i * ND + mu) * NCNC;
      v[0] += creal(u[0]) + creal(u[4]) + creal(u[8]);
      set_gauge_matrix_c(B, in, 0.15, g->fwd[i * ND + mu]);
      v[1] += re_trace_abc_dag_c(A1, u, B);
      set_gauge_matrix_c(B, in, 0.30, g->fwd[i * ND + mu]);
      v[2] += re_trace_abc_dag_c(A2, u, B);
    }
    for (int n = 0; n < LINE_NSTEPS; n++) kahan_add(&red[n], &c[n], v[n]);
  }
}

/* line_search_Landau (src/Gfix/line_search.c:274-341) */
static void line_search_landau(cpx *U, cpx *const *in, const geom_t *g,
                               double *red) {
  landau_probes(U, in, g, red);
  double val[LINE_NSTEPS];
  for (int j = 0; j < LINE_NSTEPS; j++) val[j] = -red[j];
  const double al[LINE_NSTEPS] = {0.0, 0.15, 0.30};
  egauge_landau(U, in, orc_approx_minimum(al, val), g);
}

static double functional_of(const cpx *U, size_t V) {
  double re = 0.0;
  for (size_t i = 0; i < V; i++)
    for (int mu = 0; mu < ND; mu++) {
      const cpx *u = U + (i * ND + mu) * NCNC;
      re += creal(u[0]) + creal(u[4]) + creal(u[8]);
    }
  return 1.0 - re / (double)(ND * NC * V);
}

/* ------------------------------------------------------------------ */
/* Landau solvers                                                      */

/* GLU's per-thread reduction slots for one thread: the three line-search
 * probes, insum, sum_conj and tr(dA dA) (src/Gfix/FACG.c:50,141-142,175) */
typedef struct {
  double ls[LINE_NSTEPS];
  double insum, conj, tr;
} red_t;

typedef struct {
  double *theta, *func;
  size_t cap, len;
} traj_t;

static void traj_push(traj_t *t, double th, const cpx *U, size_t V) {
  if (!t || t->len >= t->cap) return;
  t->theta[t->len] = th;
  if (t->func) t->func[t->len] = functional_of(U, V);
  t->len++;
}

typedef struct {
  geom_t g;
  cpx *U;
  cpx *in[NF], *sn[NF], *old[NF];
  fa_t fa;
  double alpha;
  int sd_fixed;
  red_t red;
  traj_t *traj;
} landau_t;

/* steep_Landau_FA (src/Gfix/FACG.c:181-199): derivative, FA, SD step */
static double landau_sd_step(landau_t *L) {
  const double norm = 1. / (double)(NC * L->g.V);
  const double fresh = fa_deriv(L->in, L->U, &L->g);
  L->red.tr += fresh; /* a continuation starts from the previous slots */
  traj_push(L->traj, fresh * norm, L->U, L->g.V);
  fa_apply(&L->fa);
  if (L->sd_fixed)
    egauge_landau(L->U, L->in, L->alpha, &L->g);
  else
    line_search_landau(L->U, L->in, &L->g, L->red.ls);
  return L->red.tr * norm;
}

/* steep_Landau_FACG (src/Gfix/FACG.c:238-337) */
static size_t landau_facg_run(landau_t *L, double *tr, double acc,
                              size_t max_iters) {
  const size_t V = L->g.V;
  const double norm = 1. / (double)(NC * V);
  size_t loc_iters = 0;
  *tr = landau_sd_step(L);
  for (int k = 0; k < NF; k++) {
    memcpy(L->sn[k], L->in[k], sizeof(cpx) * V);
    memcpy(L->old[k], L->in[k], sizeof(cpx) * V);
  }
  sum_der3(L->in, V, &L->red.insum);
  double inold = L->red.insum;
  for (;;) {
    memset(&L->red, 0, sizeof(L->red));
    L->red.tr += fa_deriv(L->in, L->U, &L->g);
    *tr = L->red.tr * norm;
    traj_push(L->traj, *tr, L->U, V);
    fa_apply(&L->fa);
    sum_pr3(L->in, L->old, V, &L->red.insum, &L->red.conj);
    const double insum = L->red.insum, sum_conj = L->red.conj;
    double beta = (sum_conj / inold < 0.0) ? 0.0 : sum_conj / inold; /* PRfmax */
    if (*tr < CG_TOL) beta = insum / inold;
    inold = insum;
    for (int k = 0; k < NF; k++)
      for (size_t j = 0; j < V; j++) {
        L->sn[k][j] = L->in[k][j] + beta * L->sn[k][j];
        L->old[k][j] = L->in[k][j];
      }
    if (*tr > CG_TOL)
      line_search_landau(L->U, L->sn, &L->g, L->red.ls);
    else
      egauge_landau(L->U, L->sn, L->alpha, &L->g);
    loc_iters++;
    if (!((*tr > acc) && (loc_iters < max_iters))) break;
  }
  return loc_iters;
}

/* steep_Landau_FASD (src/Gfix/FACG.c:202-235) */
static size_t landau_fasd_run(landau_t *L, double *tr, double acc,
                              size_t max_iters) {
  size_t loc_iters = 0;
  for (;;) {
    memset(&L->red, 0, sizeof(L->red));
    *tr = landau_sd_step(L);
    loc_iters++;
    if (!((*tr > acc) && (loc_iters < max_iters))) break;
  }
  return loc_iters;
}

double orc_theta_test_lin(const double *links, const size_t dims[4]) {
  geom_t g;
  if (geom_init(&g, dims)) return NAN;
  cpx *f[NF];
  for (int k = 0; k < NF; k++) f[k] = (cpx *)malloc(sizeof(cpx) * g.V);
  /* same local trace; theta_test_lin = 2 sum / (NC V) (gftests.c:214-250) */
  const double s = fa_deriv(f, (const cpx *)links, &g);
  for (int k = 0; k < NF; k++) free(f[k]);
  const double V = (double)g.V;
  geom_free(&g);
  return 2. * s / (NC * V);
}

size_t orc_landau_fa(double *links, const size_t dims[4], double gf_alpha,
                     double acc, size_t max_iters, int algo,
                     int sd_fixed_step, double *theta, double *traj_theta,
                     double *traj_func, size_t traj_cap, size_t *traj_len) {
  traj_t T = {traj_theta, traj_func, traj_cap, 0};
  if (traj_len) *traj_len = 0;
  /* FACG.c:349-353 early exit on the theta_test_lin measure */
  *theta = orc_theta_test_lin(links, dims);
  if (*theta < acc) return 0;
  landau_t L;
  memset(&L, 0, sizeof(L));
  if (geom_init(&L.g, dims)) return 0;
  const size_t V = L.g.V;
  L.U = (cpx *)links;
  L.alpha = gf_alpha;
  L.sd_fixed = sd_fixed_step;
  L.traj = traj_theta ? &T : NULL;
  for (int k = 0; k < NF; k++) {
    L.in[k] = (cpx *)fftw_malloc(sizeof(cpx) * V);
    L.sn[k] = (cpx *)calloc(V, sizeof(cpx));
    L.old[k] = (cpx *)calloc(V, sizeof(cpx));
  }
  fa_init(&L.fa, L.in, dims, ND);
  size_t iters = 0;
  if (algo == 0) {
    /* FACG (src/Gfix/FACG.c:361-384) */
    for (;;) {
      const size_t loc = landau_facg_run(&L, theta, acc, max_iters);
      iters = loc;
      if (loc >= max_iters) {
        if (*theta < 1E3 * acc) continue; /* continuation run */
        iters = ORC_SENTINEL;
      }
      break;
    }
  } else {
    /* FASD (src/Gfix/FACG.c:415-439) */
    for (;;) {
      size_t loc = landau_fasd_run(&L, theta, acc, max_iters);
      if (loc >= max_iters) {
        if (*theta < 1E3 * acc) continue;
        iters = ORC_SENTINEL;
      }
      iters += loc;
      break;
    }
  }
  fa_free(&L.fa);
  for (int k = 0; k < NF; k++) {
    fftw_free(L.in[k]);
    free(L.sn[k]);
    free(L.old[k]);
  }
  geom_free(&L.g);
  if (traj_len) *traj_len = T.len;
  return iters;
}

/* ------------------------------------------------------------------ */
/* Coulomb                                                             */

typedef struct {
  geom_t g;   /* 4D lattice */
  cpx *U;
  size_t Lcu, T;
  size_t *sfwd, *sbck;      /* [Lcu][3] in-slice neighbours */
  size_t *db0;              /* colour-0 sites when 2 colours */
  size_t ndb0;
  int ncolors;
  cpx *in[NF], *sn[NF], *old[NF];
  fa_t fa;
  double alpha;
  int sd_fixed;
  double red[LINE_NSTEPS + 2];
  traj_t *traj;
  uint64_t rng;
} coul_t;

/* draughtboard colour (src/Geometry/draughtboard.c:51-70, 3 colours) */
static size_t cb_colour(size_t i, const size_t *dims) {
  size_t even = 0, odd = 0, r = i;
  for (int mu = 0; mu < ND - 1; mu++) {
    const size_t n = r % dims[mu];
    r /= dims[mu];
    if ((dims[mu] & 1) == 0)
      even += n;
    else
      odd += n;
  }
  return (even % 2 + odd) % 3;
}

/* steep_deriv_CG (src/Gfix/CFACG.c:91-163) */
static void coul_deriv(coul_t *C, cpx *const *gauge, size_t t) {
  for (size_t i = 0; i < C->Lcu; i++) {
    cpx sum[5] = {0, 0, 0, 0, 0}, A[5], B[5], Cm[9], D[9];
    const size_t Uidx = i + C->Lcu * t;
    for (int mu = 0; mu < ND - 1; mu++) {
      const size_t Ubck = C->g.bck[Uidx * ND + mu];
      const size_t bck = C->sbck[i * 3 + mu], it = C->sfwd[i * 3 + mu];
      memcpy(Cm, C->U + (Uidx * ND + mu) * NCNC, sizeof(Cm));
      gtransform_local_c(gauge[i], Cm, gauge[it]);
      memcpy(D, C->U + (Ubck * ND + mu) * NCNC, sizeof(D));
      gtransform_local_c(gauge[bck], D, gauge[i]);
      hermitian_proj_short_c(B, Cm);
      hermitian_proj_short_c(A, D);
      for (int k = 0; k < 5; k++) sum[k] += A[k] - B[k];
    }
    C->in[0][i] = I * creal(sum[0]) - creal(sum[3]);
    C->in[1][i] = I * creal(sum[1]) - cimag(sum[1]);
    C->in[2][i] = I * creal(sum[2]) - cimag(sum[2]);
    C->in[3][i] = I * creal(sum[4]) - cimag(sum[4]);
  }
}

/* sum_DER2 (src/Gfix/CFACG.c:165-202), Kahan onto red[3] */
static void coul_sum_der(coul_t *C) {
  double c = 0.0;
  for (size_t i = 0; i < C->Lcu; i++) {
    double l = 0.0;
    const double a = creal(C->in[0][i]), b = cimag(C->in[0][i]);
    l += a * a + b * b + a * b;
    for (int k = 1; k < NF; k++)
      l += creal(C->in[k][i]) * creal(C->in[k][i]) +
           cimag(C->in[k][i]) * cimag(C->in[k][i]);
    kahan_add(&C->red[LINE_NSTEPS], &c, 2 * l);
  }
}

/* sum_PR (src/Gfix/CFACG.c:204-258), Kahan onto red[3], red[4] */
static void coul_sum_pr(coul_t *C) {
  double c0 = 0.0, c1 = 0.0;
  for (size_t i = 0; i < C->Lcu; i++) {
    double l1 = 0.0, l2 = 0.0;
    const double a = creal(C->in[0][i]), b = cimag(C->in[0][i]);
    l1 += a * a + b * b + a * b;
    for (int k = 1; k < NF; k++)
      l1 += creal(C->in[k][i]) * creal(C->in[k][i]) +
            cimag(C->in[k][i]) * cimag(C->in[k][i]);
    cpx t = C->in[0][i] - C->old[0][i];
    l2 += 2.0 * (a * creal(t) + b * cimag(t));
    l2 += a * cimag(t) + b * creal(t);
    for (int k = 1; k < NF; k++) {
      t = C->in[k][i] - C->old[k][i];
      l2 += 2.0 * (creal(C->in[k][i]) * creal(t) +
                   cimag(C->in[k][i]) * cimag(t));
    }
    kahan_add(&C->red[LINE_NSTEPS], &c0, 2 * l1);
    kahan_add(&C->red[LINE_NSTEPS + 1], &c1, l2);
  }
}

/* exponentiate_gauge_CG (src/Gfix/line_search.c:101-115) */
static void coul_exponentiate(coul_t *C, cpx **gauge, cpx *const *in,
                              double alpha) {
  for (size_t i = 0; i < C->Lcu; i++) {
    cpx tmp[9], tmp2[9];
    set_gauge_matrix_c(tmp, in, alpha, i);
    memcpy(tmp2, gauge[i], sizeof(tmp2));
    multab_suNC_c(gauge[i], tmp, tmp2);
  }
}

/* line_search_Coulomb / CoulombOdd + line_exp
 * (src/Gfix/line_search.c:119-271); probes 0, 0.17, 0.34 */
static void coul_line_search(coul_t *C, cpx **gauge, cpx *const *in,
                             size_t t) {
  const double PC1 = 0.17, PC2 = 0.34;
  double c[LINE_NSTEPS] = {0., 0., 0.};
  double *red = C->red;
  if (C->ncolors != 2) {
    for (size_t i = 0; i < C->Lcu; i++) {
      cpx A1[9], A2[9], B[9], Cm[9];
      double v[LINE_NSTEPS] = {0., 0., 0.};
      set_gauge_matrix_c(A1, in, PC1, i);
      set_gauge_matrix_c(A2, in, PC2, i);
      for (int mu = 0; mu < ND - 1; mu++) {
        const size_t fwd = C->sfwd[i * 3 + mu];
        memcpy(Cm, C->U + ((i + C->Lcu * t) * ND + mu) * NCNC, sizeof(Cm));
        gtransform_local_c(gauge[i], Cm, gauge[fwd]);
        v[0] += creal(Cm[0] + Cm[4] + Cm[8]);
        set_gauge_matrix_c(B, in, PC1, fwd);
        v[1] += re_trace_abc_dag_c(A1, Cm, B);
        set_gauge_matrix_c(B, in, PC2, fwd);
        v[2] += re_trace_abc_dag_c(A2, Cm, B);
      }
      for (int n = 0; n < LINE_NSTEPS; n++) kahan_add(&red[n], &c[n], v[n]);
    }
  } else {
    for (size_t s = 0; s < C->ndb0; s++) {
      const size_t idx = C->db0[s];
      cpx A1[9], A2[9], B[9], Cm[9], D[9];
      double v[LINE_NSTEPS] = {0., 0., 0.};
      set_gauge_matrix_c(A1, in, PC1, idx);
      set_gauge_matrix_c(A2, in, PC2, idx);
      for (int mu = 0; mu < ND - 1; mu++) {
        const size_t fwd = C->sfwd[idx * 3 + mu], bck = C->sbck[idx * 3 + mu];
        memcpy(Cm, C->U + ((idx + C->Lcu * t) * ND + mu) * NCNC, sizeof(Cm));
        gtransform_local_c(gauge[idx], Cm, gauge[fwd]);
        memcpy(D, C->U + ((bck + C->Lcu * t) * ND + mu) * NCNC, sizeof(D));
        gtransform_local_c(gauge[bck], D, gauge[idx]);
        v[0] += creal(Cm[0] + Cm[4] + Cm[8]);
        v[0] += creal(D[0] + D[4] + D[8]);
        set_gauge_matrix_c(B, in, PC1, fwd);
        v[1] += re_trace_abc_dag_c(A1, Cm, B);
        set_gauge_matrix_c(B, in, PC1, bck);
        v[1] += re_trace_abc_dag_c(B, D, A1);
        set_gauge_matrix_c(B, in, PC2, fwd);
        v[2] += re_trace_abc_dag_c(A2, Cm, B);
        set_gauge_matrix_c(B, in, PC2, bck);
        v[2] += re_trace_abc_dag_c(B, D, A2);
      }
      for (int n = 0; n < LINE_NSTEPS; n++) kahan_add(&red[n], &c[n], v[n]);
    }
  }
  double val[LINE_NSTEPS];
  for (int j = 0; j < LINE_NSTEPS; j++) val[j] = -red[j];
  const double al[LINE_NSTEPS] = {0.0, PC1, PC2};
  coul_exponentiate(C, gauge, in, orc_approx_minimum(al, val));
}

static double coul_theta(const coul_t *C) {
  return C->red[LINE_NSTEPS] / (double)(NC * C->Lcu);
}

static void coul_traj(coul_t *C, double th) {
  traj_t *t = C->traj;
  if (!t || t->len >= t->cap) return;
  t->theta[t->len++] = th;
}

/* steep_step_FACG (src/Gfix/CFACG.c:285-381) */
static size_t coul_facg_run(coul_t *C, cpx **gauge, double *tr, size_t t,
                            double acc, size_t max_iters) {
  const double norm = 1. / (double)(NC * C->Lcu);
  size_t loc_iters = 0;
  memset(C->red, 0, sizeof(C->red));
  coul_deriv(C, gauge, t);
  fa_apply(&C->fa);
  coul_sum_der(C);
  double inold = C->red[LINE_NSTEPS];
  *tr = inold * norm;
  coul_traj(C, *tr);
  coul_line_search(C, gauge, C->in, t);
  for (int k = 0; k < NF; k++) {
    memcpy(C->sn[k], C->in[k], sizeof(cpx) * C->Lcu);
    memcpy(C->old[k], C->in[k], sizeof(cpx) * C->Lcu);
  }
  for (;;) {
    memset(C->red, 0, sizeof(C->red));
    coul_deriv(C, gauge, t);
    fa_apply(&C->fa);
    coul_sum_pr(C);
    const double insum = C->red[LINE_NSTEPS], sum_conj = C->red[LINE_NSTEPS + 1];
    *tr = insum * norm;
    coul_traj(C, *tr);
    double beta = (sum_conj / inold < 0.0) ? 0.0 : sum_conj / inold;
    if (*tr < CG_TOL) beta = insum / inold;
    inold = insum;
    for (int k = 0; k < NF; k++)
      for (size_t j = 0; j < C->Lcu; j++) {
        C->sn[k][j] = C->in[k][j] + beta * C->sn[k][j];
        C->old[k][j] = C->in[k][j];
      }
    if (*tr > CG_TOL)
      coul_line_search(C, gauge, C->sn, t);
    else
      coul_exponentiate(C, gauge, C->sn, C->alpha);
    loc_iters++;
    if (!((*tr > acc) && (loc_iters < max_iters))) break;
  }
  return loc_iters;
}

/* steep_step_FASD (src/Gfix/CFACG.c:384-429) */
static size_t coul_fasd_run(coul_t *C, cpx **gauge, double *tr, size_t t,
                            double acc, size_t max_iters) {
  size_t loc_iters = 0;
  for (;;) {
    memset(C->red, 0, sizeof(C->red));
    coul_deriv(C, gauge, t);
    fa_apply(&C->fa);
    if (C->sd_fixed)
      coul_exponentiate(C, gauge, C->in, C->alpha);
    else
      coul_line_search(C, gauge, C->in, t);
    coul_sum_der(C);
    *tr = coul_theta(C);
    coul_traj(C, *tr);
    loc_iters++;
    if (!((*tr > acc) && (loc_iters < max_iters))) break;
  }
  return loc_iters;
}

/* a unitary matrix from our own generator; the reference's Sunitary_gen
 * stream (src/Utils/par_rng.c) is not reproduced, so restarted slices are
 * never compared value for value */
static double rng_uniform(uint64_t *s) {
  *s = *s * 6364136223846793005ull + 1442695040888963407ull;
  return ((*s >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static void random_su3(cpx *u, uint64_t *s) {
  for (int k = 0; k < 9; k++) {
    const double r1 = rng_uniform(s), r2 = rng_uniform(s);
    const double rad = sqrt(-2.0 * log(r1));
    u[k] = rad * cos(TWOPI_GLU * r2) + I * rad * sin(TWOPI_GLU * r2);
  }
  gram_reunit_c(u);
}

/* adequate_solution (src/Gfix/CFACG.c:432-456): reunitarise g and check
 * the norm; returns 1 when adequate */
static int coul_adequate(coul_t *C, cpx **gauge, size_t iters) {
  int ok = 1;
  for (size_t i = 0; i < C->Lcu; i++) {
    gram_reunit_c(gauge[i]);
    double s = 0.0;
    for (int j = 0; j < NCNC; j++)
      s += creal(gauge[i][j]) * creal(gauge[i][j]) +
           cimag(gauge[i][j]) * cimag(gauge[i][j]);
    if (fabs(s - NC) > (double)iters * PREC_TOL) ok = 0;
  }
  return ok;
}

/* steep_fix (src/Gfix/CFACG.c:459-529) */
static size_t coul_steep_fix(coul_t *C, cpx **gauge, size_t t, double acc,
                             size_t max_iters, int facg, double *tr_out,
                             size_t *restarts) {
  double tr = 1.0;
  size_t tot = 0, control = 0;
  int trans = 0;
  for (;;) {
    const size_t loc = facg ? coul_facg_run(C, gauge, &tr, t, acc, max_iters)
                            : coul_fasd_run(C, gauge, &tr, t, acc, max_iters);
    if (tr < acc)
      if (!coul_adequate(C, gauge, loc > 0 ? loc : 1)) trans = 1;
    if (loc >= max_iters) {
      if (tr < 1E4 * acc && !isnan(tr) && !isinf(tr)) {
        tot += loc;
        continue;
      }
      if (tr > acc || isnan(tr) || isinf(tr)) trans = 1;
    }
    if (control < 8 && trans) {
      for (size_t i = 0; i < C->Lcu; i++) random_su3(gauge[i], &C->rng);
      tot += loc;
      control++;
      if (restarts) (*restarts)++;
      trans = 0;
      continue;
    }
    tot += loc;
    break;
  }
  *tr_out = tr;
  return tot;
}

/* gtransform_slice (src/Gfix/gtrans.c:214-238) */
static void coul_slice_transform(coul_t *C, cpx **g, cpx **gup, size_t t) {
  for (size_t i = 0; i < C->Lcu; i++) {
    const size_t j = C->Lcu * t + i;
    for (int mu = 0; mu < ND - 1; mu++)
      gtransform_local_c(g[i], C->U + (j * ND + mu) * NCNC,
                         g[C->sfwd[i * 3 + mu]]);
    gtransform_local_c(g[i], C->U + (j * ND + ND - 1) * NCNC, gup[i]);
  }
}

size_t orc_coulomb_fa(double *links, const size_t dims[4], double gf_alpha,
                      double acc, size_t max_iters, int facg,
                      int sd_fixed_step, double *slice_theta,
                      size_t *slice_iters, double *traj_theta,
                      size_t traj_cap, size_t *traj_len, size_t *restarts) {
  traj_t Tr = {traj_theta, NULL, traj_cap, 0};
  coul_t C;
  memset(&C, 0, sizeof(C));
  if (geom_init(&C.g, dims)) return 0;
  C.U = (cpx *)links;
  C.Lcu = dims[0] * dims[1] * dims[2];
  C.T = dims[3];
  C.alpha = gf_alpha;
  C.sd_fixed = sd_fixed_step;
  C.traj = traj_theta ? &Tr : NULL;
  C.rng = 0x9E3779B97F4A7C15ull;
  if (restarts) *restarts = 0;
  C.sbck = (size_t *)malloc(sizeof(size_t) * C.Lcu * 3);
  /* for i < Lcu the three spatial neighbours stay in slice t = 0 */
  size_t *sf = (size_t *)malloc(sizeof(size_t) * C.Lcu * 3);
  for (size_t i = 0; i < C.Lcu; i++)
    for (int mu = 0; mu < 3; mu++) {
      sf[i * 3 + mu] = C.g.fwd[i * ND + mu];
      C.sbck[i * 3 + mu] = C.g.bck[i * ND + mu];
    }
  C.sfwd = sf;
  /* init_cb (src/Geometry/draughtboard.c:76-128) */
  size_t ncol[3] = {0, 0, 0};
  for (size_t i = 0; i < C.Lcu; i++) ncol[cb_colour(i, dims)]++;
  C.ncolors = ncol[2] == 0 ? 2 : 3;
  C.db0 = (size_t *)malloc(sizeof(size_t) * (ncol[0] ? ncol[0] : 1));
  for (size_t i = 0; i < C.Lcu; i++)
    if (cb_colour(i, dims) == 0) C.db0[C.ndb0++] = i;
  for (int k = 0; k < NF; k++) {
    C.in[k] = (cpx *)fftw_malloc(sizeof(cpx) * C.Lcu);
    C.sn[k] = (cpx *)calloc(C.Lcu, sizeof(cpx));
    C.old[k] = (cpx *)calloc(C.Lcu, sizeof(cpx));
  }
  fa_init(&C.fa, C.in, dims, ND - 1);
  cpx **G[3];
  for (int k = 0; k < 3; k++) {
    G[k] = (cpx **)malloc(sizeof(cpx *) * C.Lcu);
    for (size_t i = 0; i < C.Lcu; i++) {
      G[k][i] = (cpx *)malloc(sizeof(cpx) * 9);
      identity_c(G[k][i]);
    }
  }
  cpx **g_end = G[0], **g = G[1], **g_up = G[2];
  /* Coulomb_FA slice order (src/Gfix/CFACG.c:572-619) */
  size_t tot = 0, t;
  double th;
  {
    const size_t it0 =
        coul_steep_fix(&C, g_end, 0, acc, max_iters, facg, &th, restarts);
    if (slice_iters) slice_iters[0] = it0;
    if (slice_theta) slice_theta[0] = th;
    tot += it0;
    const size_t it1 =
        coul_steep_fix(&C, g, 1, acc, max_iters, facg, &th, restarts);
    if (slice_iters) slice_iters[1] = it1;
    if (slice_theta) slice_theta[1] = th;
    tot += it1;
  }
  coul_slice_transform(&C, g_end, g, 0);
  for (t = 2; t < C.T; t++) {
    for (size_t i = 0; i < C.Lcu; i++) identity_c(g_up[i]);
    const size_t it =
        coul_steep_fix(&C, g_up, t, acc, max_iters, facg, &th, restarts);
    if (slice_iters) slice_iters[t] = it;
    if (slice_theta) slice_theta[t] = th;
    tot += it;
    coul_slice_transform(&C, g, g_up, t - 1);
    cpx **p = g;
    g = g_up;
    g_up = p;
  }
  coul_slice_transform(&C, g, g_end, t - 1);
  for (int k = 0; k < 3; k++) {
    for (size_t i = 0; i < C.Lcu; i++) free(G[k][i]);
    free(G[k]);
  }
  fa_free(&C.fa);
  for (int k = 0; k < NF; k++) {
    fftw_free(C.in[k]);
    free(C.sn[k]);
    free(C.old[k]);
  }
  free(C.db0);
  free(C.sbck);
  free(sf);
  geom_free(&C.g);
  if (traj_len) *traj_len = Tr.len;
  return tot;
}

/* ------------------------------------------------------------------ */
/* single pieces                                                       */

double orc_gauge_functional(const double *links, const size_t dims[4]) {
  size_t V = dims[0] * dims[1] * dims[2] * dims[3];
  return functional_of((const cpx *)links, V);
}

/* average plaquette (src/Field/plaqs_links.c:243-265) */
double orc_plaquette(const double *links, const size_t dims[4]) {
  geom_t g;
  if (geom_init(&g, dims)) return NAN;
  const cpx *U = (const cpx *)links;
  double plaq = 0.0;
  for (size_t i = 0; i < g.V; i++) {
    double p = 0.0;
    for (int mu = 0; mu < ND; mu++) {
      const size_t tt = g.fwd[i * ND + mu];
      for (int nu = 0; nu < mu; nu++) {
        const size_t s = g.fwd[i * ND + nu];
        const cpx *a = U + (i * ND + mu) * NCNC, *b = U + (tt * ND + nu) * NCNC;
        const cpx *c = U + (s * ND + mu) * NCNC, *d = U + (i * ND + nu) * NCNC;
        /* Re tr(a b c^dag d^dag) */
        cpx ab[9], dc[9];
        for (int r = 0; r < 3; r++)
          for (int k = 0; k < 3; k++) {
            cpx s1 = 0, s2 = 0;
            for (int j = 0; j < 3; j++) {
              s1 += a[r * 3 + j] * b[j * 3 + k];
              s2 += d[r * 3 + j] * c[j * 3 + k];
            }
            ab[r * 3 + k] = s1;
            dc[r * 3 + k] = s2;
          }
        double tr = 0.0;
        for (int k = 0; k < 9; k++) tr += creal(ab[k] * conj(dc[k]));
        p += tr;
      }
    }
    plaq += p;
  }
  const double V = (double)g.V;
  geom_free(&g);
  return 2.0 * plaq / (NC * ND * (ND - 1) * V);
}

void orc_reunit_links(double *links, size_t nlinks) {
  for (size_t l = 0; l < nlinks; l++) gram_reunit_c((cpx *)links + l * NCNC);
}

double orc_derivative(const double *links, const size_t dims[4],
                      double *fields) {
  geom_t g;
  if (geom_init(&g, dims)) return NAN;
  cpx *f[NF];
  for (int k = 0; k < NF; k++) f[k] = (cpx *)fields + (size_t)k * g.V;
  const double s = fa_deriv(f, (const cpx *)links, &g);
  const double V = (double)g.V;
  geom_free(&g);
  return s / (NC * V);
}

void orc_fourier_accelerate(double *fields, const size_t dims[4], int ndim) {
  size_t vol = 1;
  for (int mu = 0; mu < ndim; mu++) vol *= dims[mu];
  cpx *f[NF];
  for (int k = 0; k < NF; k++) {
    f[k] = (cpx *)fftw_malloc(sizeof(cpx) * vol);
    memcpy(f[k], (cpx *)fields + (size_t)k * vol, sizeof(cpx) * vol);
  }
  fa_t fa;
  fa_init(&fa, f, dims, ndim);
  fa_apply(&fa);
  for (int k = 0; k < NF; k++) {
    memcpy((cpx *)fields + (size_t)k * vol, f[k], sizeof(cpx) * vol);
    fftw_free(f[k]);
  }
  fa_free(&fa);
}

void orc_dft(double *data, int rank, const int *n, int sign) {
  fftw_plan p = fftw_plan_dft(rank, n, (fftw_complex *)data,
                              (fftw_complex *)data, sign, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
}

void orc_sum_pr(const double *in, const double *in_old, size_t V,
                double *out) {
  cpx *a[NF], *b[NF];
  for (int k = 0; k < NF; k++) {
    a[k] = (cpx *)in + (size_t)k * V;
    b[k] = (cpx *)in_old + (size_t)k * V;
  }
  out[0] = out[1] = 0.0;
  sum_pr3(a, b, V, &out[0], &out[1]);
}

double orc_line_search_probes(const double *links, const size_t dims[4],
                              const double *sn, double *val) {
  geom_t g;
  if (geom_init(&g, dims)) return NAN;
  cpx *f[NF];
  for (int k = 0; k < NF; k++) f[k] = (cpx *)sn + (size_t)k * g.V;
  double red[LINE_NSTEPS] = {0., 0., 0.};
  landau_probes((const cpx *)links, f, &g, red);
  for (int j = 0; j < LINE_NSTEPS; j++) val[j] = -red[j];
  geom_free(&g);
  const double al[LINE_NSTEPS] = {0.0, 0.15, 0.30};
  return orc_approx_minimum(al, val);
}

void orc_link_update(double *links, const size_t dims[4], const double *sn,
                     double alpha) {
  geom_t g;
  if (geom_init(&g, dims)) return;
  cpx *f[NF];
  for (int k = 0; k < NF; k++) f[k] = (cpx *)sn + (size_t)k * g.V;
  egauge_landau((cpx *)links, f, alpha, &g);
  geom_free(&g);
}

void orc_gauge_matrix(const double *fields, size_t V, size_t i, double alpha,
                      double *gout) {
  cpx *f[NF];
  for (int k = 0; k < NF; k++) f[k] = (cpx *)fields + (size_t)k * V;
  set_gauge_matrix_c((cpx *)gout, f, alpha, i);
}

void orc_gram_reunit(double *u) { gram_reunit_c((cpx *)u); }
