/*
 * Minimal FFTW3-API stand-in used only to build the CPU oracle of the
 * reference (GLU) in a container that has no libfftw3.
 *
 * Test infrastructure: nothing in the product library includes this file.
 *
 * It declares the subset of the public FFTW3 API that GLU calls
 * (src/Geometry/plan_ffts.c:79-240, src/Gfix/FACG.c:86,91,
 * src/Gfix/CFACG.c:79,84, src/Field/balls.c and the Cuts sources).  The semantics
 * follow FFTW's published conventions: row-major multi-dimensional complex
 * DFT (last dimension fastest), sign -1 forward / +1 backward, no
 * normalisation, out-of-place or in-place.  The transform itself is our own
 * mixed-radix code in fftw_shim.c.
 */
#ifndef GLU_B200_FFTW_SHIM_H
#define GLU_B200_FFTW_SHIM_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FFTW's rule: when <complex.h> came first, fftw_complex is the C99 type. */
#if defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif

typedef struct glu_shim_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in,
                        fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
void fftw_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
int fftw_import_wisdom_from_file(FILE *input_file);
int fftw_import_wisdom_from_filename(const char *filename);
void fftw_export_wisdom_to_file(FILE *output_file);
int fftw_export_wisdom_to_filename(const char *filename);

/*
 * Shim-only extension: an observer called around every fftw_execute.
 * `when` is 0 before the transform runs and 1 after it.  The oracle harness
 * uses it to record per-iteration trajectories without touching the
 * reference sources.
 */
typedef void (*glu_shim_hook_fn)(void *ctx, fftw_plan p, int when, int sign,
                                 void *in, void *out);
void glu_shim_set_hook(glu_shim_hook_fn fn, void *ctx);
/* accumulated wall time spent inside fftw_execute (seconds) */
double glu_shim_fft_seconds(void);
void glu_shim_reset_fft_seconds(void);

#ifdef __cplusplus
}
#endif

#endif
