/*
 * Our own mixed-radix complex DFT behind the FFTW3 API subset declared in
 * fftw3.h.  Test infrastructure for the CPU oracle only.
 *
 * Conventions (FFTW's published ones): a rank-r plan over dims n[0..r-1]
 * is row-major (n[r-1] fastest); FFTW_FORWARD uses exp(-2 pi i jk/N),
 * FFTW_BACKWARD exp(+2 pi i jk/N); neither direction is normalised.
 *
 * Algorithm: each axis is transformed pencil by pencil with a recursive
 * decimation-in-time mixed-radix FFT (radices 4, 2, 3, 5 and a direct DFT
 * for any other prime).  Twiddles are cos/sin of 2 pi k/N evaluated
 * directly per k, so each one is correctly rounded to within an ulp.
 */
#include "fftw3.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
  double re, im;
} cpx;

typedef struct {
  int n;
  int nfac;
  int fac[64];
  cpx *tw; /* tw[k] = exp(sign * 2 pi i k / n), k < n */
} axis_plan;

struct glu_shim_plan_s {
  int rank;
  int sign;
  int dims[16];
  size_t total;
  cpx *in, *out;
  axis_plan ax[16];
};

static glu_shim_hook_fn g_hook = NULL;
static void *g_hook_ctx = NULL;
static uint64_t g_fft_ns = 0;

void glu_shim_set_hook(glu_shim_hook_fn fn, void *ctx) {
  g_hook = fn;
  g_hook_ctx = ctx;
}

double glu_shim_fft_seconds(void) {
  return (double)__atomic_load_n(&g_fft_ns, __ATOMIC_RELAXED) * 1e-9;
}

void glu_shim_reset_fft_seconds(void) {
  __atomic_store_n(&g_fft_ns, 0, __ATOMIC_RELAXED);
}

static uint64_t now_ns(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

static void factorise(axis_plan *a) {
  int n = a->n, k = 0;
  while (n % 4 == 0) { a->fac[k++] = 4; n /= 4; }
  while (n % 2 == 0) { a->fac[k++] = 2; n /= 2; }
  for (int p = 3; n > 1; p += 2) {
    while (n % p == 0) { a->fac[k++] = p; n /= p; }
    if (p * p > n && n > 1) { a->fac[k++] = n; n = 1; }
  }
  if (k == 0) a->fac[k++] = 1;
  a->nfac = k;
}

static int axis_init(axis_plan *a, int n, int sign) {
  a->n = n;
  factorise(a);
  a->tw = (cpx *)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
  if (!a->tw) return -1;
  const double two_pi = 6.283185307179586476925286766559;
  for (int k = 0; k < n; k++) {
    const double ang = two_pi * (double)k / (double)n;
    a->tw[k].re = cos(ang);
    a->tw[k].im = (double)sign * sin(ang);
  }
  return 0;
}

static inline cpx cmul(cpx a, cpx b) {
  cpx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

/*
 * out[0..n) <- DFT_n of in[0], in[s], ..., in[(n-1)s] where n divides N and
 * the twiddle step for this level is N/n (tw is the size-N table).
 */
static void fft_rec(cpx *out, const cpx *in, size_t s, int n, const int *fac,
                    const cpx *tw, int N, cpx *tmp) {
  const int p = fac[0];
  const int m = n / p;
  if (m == 1) {
    for (int j = 0; j < p; j++) out[j] = in[(size_t)j * s];
  } else {
    for (int j = 0; j < p; j++)
      fft_rec(out + (size_t)j * m, in + (size_t)j * s, s * (size_t)p, m,
              fac + 1, tw, N, tmp);
  }
  const int step = N / n; /* W_n^q = tw[q * step] */
  if (p == 2) {
    for (int k = 0; k < m; k++) {
      cpx a = out[k];
      cpx b = cmul(out[k + m], tw[k * step]);
      out[k].re = a.re + b.re; out[k].im = a.im + b.im;
      out[k + m].re = a.re - b.re; out[k + m].im = a.im - b.im;
    }
    return;
  }
  if (p == 4) {
    /* W_4 = tw[N/4]: +-i depending on the sign stored in the table */
    const cpx w4 = tw[N / 4];
    for (int k = 0; k < m; k++) {
      cpx y0 = out[k];
      cpx y1 = cmul(out[k + m], tw[k * step]);
      cpx y2 = cmul(out[k + 2 * m], tw[2 * k * step]);
      cpx y3 = cmul(out[k + 3 * m], tw[3 * k * step]);
      cpx a0 = {y0.re + y2.re, y0.im + y2.im};
      cpx a1 = {y0.re - y2.re, y0.im - y2.im};
      cpx b0 = {y1.re + y3.re, y1.im + y3.im};
      cpx b1 = cmul((cpx){y1.re - y3.re, y1.im - y3.im}, w4);
      out[k].re = a0.re + b0.re; out[k].im = a0.im + b0.im;
      out[k + m].re = a1.re + b1.re; out[k + m].im = a1.im + b1.im;
      out[k + 2 * m].re = a0.re - b0.re; out[k + 2 * m].im = a0.im - b0.im;
      out[k + 3 * m].re = a1.re - b1.re; out[k + 3 * m].im = a1.im - b1.im;
    }
    return;
  }
  /* generic radix p: X[k + q m] = sum_j W_n^{jk} Y_j[k] W_p^{jq} */
  for (int k = 0; k < m; k++) {
    for (int j = 0; j < p; j++) {
      const size_t idx = ((size_t)j * (size_t)k * (size_t)step) % (size_t)N;
      tmp[j] = cmul(out[k + j * m], tw[idx]);
    }
    for (int q = 0; q < p; q++) {
      cpx acc = {0.0, 0.0};
      for (int j = 0; j < p; j++) {
        const size_t idx =
            ((size_t)j * (size_t)q % (size_t)p) * (size_t)(N / p);
        cpx t = cmul(tmp[j], tw[idx]);
        acc.re += t.re;
        acc.im += t.im;
      }
      out[k + q * m] = acc;
    }
  }
}

static void fft_1d(const axis_plan *a, cpx *data, size_t stride, cpx *buf,
                   cpx *tmp) {
  const int n = a->n;
  if (n <= 1) return;
  for (int j = 0; j < n; j++) buf[n + j] = data[(size_t)j * stride];
  fft_rec(buf, buf + n, 1, n, a->fac, a->tw, n, tmp);
  for (int j = 0; j < n; j++) data[(size_t)j * stride] = buf[j];
}

fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in,
                        fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  if (rank < 1 || rank > 16) return NULL;
  struct glu_shim_plan_s *p =
      (struct glu_shim_plan_s *)calloc(1, sizeof(struct glu_shim_plan_s));
  if (!p) return NULL;
  p->rank = rank;
  p->sign = sign;
  p->total = 1;
  for (int d = 0; d < rank; d++) {
    p->dims[d] = n[d];
    p->total *= (size_t)n[d];
    if (axis_init(&p->ax[d], n[d], sign) != 0) {
      fftw_destroy_plan(p);
      return NULL;
    }
  }
  p->in = (cpx *)(void *)in;
  p->out = (cpx *)(void *)out;
  return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags) {
  return fftw_plan_dft(1, &n, in, out, sign, flags);
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (g_hook) g_hook(g_hook_ctx, p, 0, p->sign, p->in, p->out);
  const uint64_t t0 = now_ns();
  if (p->out != p->in) memcpy(p->out, p->in, sizeof(cpx) * p->total);
  int nmax = 1;
  for (int d = 0; d < p->rank; d++)
    if (p->dims[d] > nmax) nmax = p->dims[d];
  cpx *buf = (cpx *)malloc(sizeof(cpx) * (size_t)(3 * nmax + 8));
  if (!buf) abort();
  cpx *tmp = buf + 2 * nmax;
  size_t stride = 1;
  for (int d = p->rank - 1; d >= 0; d--) {
    const size_t n = (size_t)p->dims[d];
    const size_t outer = p->total / (n * stride);
    for (size_t o = 0; o < outer; o++) {
      for (size_t s = 0; s < stride; s++) {
        fft_1d(&p->ax[d], p->out + o * n * stride + s, stride, buf, tmp);
      }
    }
    stride *= n;
  }
  free(buf);
  __atomic_fetch_add(&g_fft_ns, now_ns() - t0, __ATOMIC_RELAXED);
  if (g_hook) g_hook(g_hook_ctx, p, 1, p->sign, p->in, p->out);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  for (int d = 0; d < p->rank; d++) free(p->ax[d].tw);
  free(p);
}

void *fftw_malloc(size_t n) {
  void *ptr = NULL;
  if (posix_memalign(&ptr, 64, n ? n : 1) != 0) return NULL;
  return ptr;
}

void fftw_free(void *p) { free(p); }
void fftw_cleanup(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup_threads(void) {}
int fftw_import_wisdom_from_file(FILE *f) { (void)f; return 0; }
int fftw_import_wisdom_from_filename(const char *f) { (void)f; return 0; }
void fftw_export_wisdom_to_file(FILE *f) { (void)f; }
int fftw_export_wisdom_to_filename(const char *f) { (void)f; return 1; }
