/*
 * glu_gfix.h -- C ABI of the B200 (sm_100a) Fourier-accelerated gauge
 * fixing library libglu_gfix.so.
 *
 * Two layers are exported.
 *
 * 1. GLU's own gauge-fixing entry points, with GLU's signatures, so that the
 *    GLU program links against this library in place of the archive members
 *    FACG.o, Landau.o, Coulomb.o and CFACG.o.  The structs are GLU's
 *    (src/Headers/GLU_types.h) for the default build NC = 3, ND = 4, double
 *    precision, with FFTW: they are only forward-declared here, and the
 *    library reads them with that layout.  Dimensions and the tuning
 *    parameter come from GLU's global `Latt` (src/Headers/Mainfile.h:74).
 *
 * 2. A flat interface with plain pointers and sizes (gfix_*), which the
 *    GLU entry points and the Python package glu_b200 both call.
 *
 * Link layout of the flat interface: double[V][4][9][2] -- site index
 * s = x + Lx (y + Ly (z + Lz t)), then mu, then a row-major 3x3 complex
 * matrix as (re, im) -- GLU's in-memory order of lat[s].O[mu][a*3+b].
 *
 * All calls are synchronous: on return the links have been copied back.
 * A call uses the current CUDA device.  Calls are not re-entrant (GLU's are
 * not either): the library keeps one cached workspace per device and
 * lattice shape.
 *
 * Ordering of the entry points that take device pointers (the _device
 * variants, gfix_coulomb_slices*, gfix_profile_*): the library works on its
 * own non-blocking streams, so each of them first waits for all work on
 * the device (cudaDeviceSynchronize) before it reads the caller's buffers,
 * and has finished writing them when it returns.  The one exception is
 * gfix_theta_functional_noalloc, which is ordered on the stream it is given.
 */
#ifndef GLU_B200_GFIX_H
#define GLU_B200_GFIX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GLU types, by reference only (src/Headers/GLU_types.h) */
struct site;
struct fftw_stuff;
struct cut_info;

/* ---------------------------------------------------------------------
 * GLU entry points
 * ------------------------------------------------------------------- */

/* Landau gauge fixing by Fourier-accelerated non-linear CG.
 * Replaces src/Gfix/FACG.c:341-391 (declared src/Headers/FACG.h:37-41).
 * Returns the iteration count, 123456789 on non-convergence; *th receives
 * the final in-loop theta.  FFTW may be NULL: plans and p^2 live on the GPU. */
size_t FACG(struct site *lat, struct fftw_stuff *FFTW, double *th,
            const double acc, const size_t max_iters);

/* Landau gauge fixing by Fourier-accelerated steepest descent.
 * Replaces src/Gfix/FACG.c:395-446 (src/Headers/FACG.h:54-58). */
size_t FASD(struct site *lat, struct fftw_stuff *FFTW, double *th,
            const double acc, const size_t max_iters);

/* FFT, multiply by FFTW->psq, inverse FFT of the 4 packed fields
 * FFTW->in[0..3] in place, on the GPU.  Replaces src/Gfix/FACG.c:77-95. */
void FOURIER_ACCELERATE3(struct fftw_stuff *FFTW);

/* Landau driver: FA solve, up to GF_GLU_FAILURES-1 random restarts,
 * reunitarisation and the "[GF]" summary.  Replaces
 * src/Gfix/Landau.c:261-374 (src/Headers/Landau.h:51-54).  Restarts use the
 * links as they were on entry (kept on the GPU) instead of re-reading
 * `infile`, and random gauge transforms from this library's generator
 * seeded by Latt.Seed[0]; the returned count follows GLU's sums (see
 * gfix_landau), GLU_FAILURE after the last failed attempt. */
size_t Landau(struct site *lat, const double accuracy, const size_t iter,
              const char *infile);

/* Coulomb driver: all time slices solved together, slice transforms of the
 * links, final reunitarisation.  Replaces src/Gfix/Coulomb.c:32-106
 * (src/Headers/Coulomb.h:40-42). */
size_t Coulomb(struct site *lat, const double accuracy, const size_t iter);

/* Coulomb FA solve of every slice plus the slice transforms.  Replaces
 * src/Gfix/CFACG.c:531-636 (src/Headers/CFACG.h:37-41); FACG is GLU's
 * GLU_bool (0 = steepest descent, 1 = CG). */
size_t Coulomb_FA(struct site *lat, struct fftw_stuff *FFTW,
                  const double accuracy, const size_t max_iter, const int FACG);

/* 3D version of FOURIER_ACCELERATE3 over one slice of Lx*Ly*Lz sites.
 * Replaces src/Gfix/CFACG.c:69-88. */
void FOURIER_ACCELERATE2(struct fftw_stuff *FFTW);

/* Momentum-space gluon measurements: CUTTYPE = GLUON_PROPS, EXCEPTIONAL or
 * FIELDS, either field definition, every momentum cut.  Replaces
 * src/Cuts/cuts.c:110-184 (src/Headers/cuts.h:40-42): writes GLU's output
 * file into the working directory (named by output_str_struct, configuration
 * number Latt.flow) and returns GLU_SUCCESS (0), or GLU_FAILURE (-1) for
 * the other modes.  A is left unchanged. */
int cuts_struct(struct site *A, const struct cut_info CUTINFO);

/* ---------------------------------------------------------------------
 * flat interface
 * ------------------------------------------------------------------- */

enum gfix_algo { GFIX_CG = 0, GFIX_SD = 1 };
/* GFIX_MIXED: FP32 links, fields and FFT until theta < switch_theta (or a
 * stall of the FP32 run), then FP64 links, theta and updates to the
 * requested accuracy with the search directions and their Fourier
 * acceleration in FP32 (their relative precision is all a descent
 * direction needs).  GFIX_PROFILE_POLISH: gfix_profile_landau only, the
 * kernels of that second phase. */
enum gfix_precision { GFIX_FP64 = 0, GFIX_MIXED = 1, GFIX_PROFILE_POLISH = 2 };

typedef struct gfix_params {
  double gf_alpha;       /* GLU's GF_TUNE (Latt.gf_alpha)                  */
  double accuracy;       /* stop when theta < accuracy (10^-ACCURACY)      */
  size_t max_iters;      /* GLU's MAX_ITERS                                */
  int algo;              /* GFIX_CG (FACG) or GFIX_SD (FASD)               */
  int sd_fixed_step;     /* 1: GLU built with GLU_GFIX_SD (fixed step)     */
  int precision;         /* GFIX_FP64 or GFIX_MIXED                        */
  double switch_theta;   /* MIXED: FP32 until theta < switch_theta         */
  double *traj_theta;    /* optional host arrays, one entry per derivative */
  double *traj_func;     /*   evaluation (theta, gauge functional)         */
  size_t traj_cap;
  int max_restarts;      /* Landau: random restarts after a failed solve   */
                         /*   (0: none, as GLU's FACG/FASD; GLU's Landau   */
                         /*   driver makes GF_GLU_FAILURES - 1 = 6)        */
  uint64_t restart_seed; /* seed of the restarts' random gauge transforms  */
  int luxury_copies;     /* Landau: GLU's LUXURY_GAUGE copies (0: none)     */
  int luxury_best;       /* 1: keep the copy of least functional (BEST_COPY)*/
} gfix_params;

typedef struct gfix_result {
  size_t iters;          /* GLU's return value (123456789 if failed)       */
  size_t iters_fp32;     /* MIXED: iterations spent in FP32                */
  double theta;          /* final in-loop theta                            */
  size_t traj_len;
  double gpu_ms;         /* device time of the solve (CUDA events)         */
  int restarts;          /* random restarts made (Landau: max_restarts;    */
                         /*   Coulomb: over all slices; also a mixed       */
                         /*   phase restarted in FP64)                     */
} gfix_result;

/* Landau FA gauge fixing of host links (double[V][4][9][2]) in place.
 * dims = {Lx, Ly, Lz, Lt}.  Returns 0, or a negative error code (see
 * gfix_last_error).
 *
 * With p->max_restarts = 0 the result is GLU's FACG / FASD
 * (src/Gfix/FACG.c:341-446): r->iters is the iteration count, or the
 * sentinel 123456789 when the solve did not converge.  With max_restarts >
 * 0 a failed solve is retried as GLU's Landau driver does
 * (src/Gfix/Landau.c:303-340): the links as they were on entry (kept on the
 * GPU; GLU re-reads its input file), a random SU(3) gauge transform
 * (seeded by restart_seed and the attempt; GLU's random_transform draws
 * from its own generator), a new solve -- up to max_restarts times.
 * r->iters then follows GLU's accounting: the first attempt's sentinel,
 * plus max_iters per failed restart, plus the successful attempt's count;
 * (size_t)-1 (GLU_FAILURE) when every attempt failed, the links then being
 * the last attempt's.  r->restarts counts the restarts made.
 *
 * With p->luxury_copies = N > 0 each attempt is GLU's luxury_copy_fast
 * (src/Gfix/Landau.c:92-211, a LUXURY_GAUGE build): N random gauge copies
 * of the attempt's start (this library's generator), each fixed to theta <
 * 1e-6 in at most 1000 iterations; of the copies that converged within that
 * bound the one with the largest gauge functional is kept (GLU's default;
 * the smallest with p->luxury_best, GLU's BEST_COPY) and fixed to
 * p->accuracy.  r->iters is then GLU's sum: the last copy's iterations plus
 * the final fix's.  If no copy is kept the final fix starts from the
 * attempt's start.  Batches ignore both restarts and copies. */
int gfix_landau(double *links, const size_t dims[4], const gfix_params *p,
                gfix_result *r);

/* n configurations of one lattice shape fixed one after another, exactly as
 * n gfix_landau calls would fix them (results r[0..n-1], links[i] written
 * back in place), through one set of device workspaces: while
 * configuration i is solved, the links of configuration i+1 cross to the
 * device and those of i-1 back on a copy stream.  The copies overlap the
 * solves when the host arrays are pinned (cudaHostAlloc, cudaHostRegister);
 * from pageable memory the results are the same, the overlap is lost.  A
 * trajectory, when asked for, is the last configuration's.  n = 0 does
 * nothing.  No reference counterpart: GLU's program fixes one
 * configuration per run. */
int gfix_landau_sequence(double *const *links, size_t n, const size_t dims[4],
                         const gfix_params *p, gfix_result *r);

/* GLU's Landau driver (src/Gfix/Landau.c:261-374) as one device-resident
 * sequence: gfix_landau (with p->max_restarts random restarts; Landau()
 * passes GF_GLU_FAILURES - 1 = 6) and, when it converged, output_fixing_info
 * (Landau.c:42-66): the links reunitarised (latt_reunitU), then obs[0..2] as
 * gfix_observables and diag[0..5] as gfix_link_diagnostics of the result.
 * The links cross PCIe once each way.  On failure (r->iters = (size_t)-1,
 * or the sentinel with max_restarts = 0) the links are the last attempt's,
 * not reunitarised, and obs / diag are zero.  obs, diag may be NULL. */
int gfix_landau_driver(double *links, const size_t dims[4], const gfix_params *p,
                       gfix_result *r, double *obs, double *diag);

/* GLU's Coulomb driver (src/Gfix/Coulomb.c:32-106) as one device-resident
 * sequence: obs_in / diag_in of the input (GLU prints the initial link
 * traces and plaquette), gfix_coulomb, latt_reunitU, obs / diag of the
 * result (layouts as gfix_observables / gfix_link_diagnostics; each may be
 * NULL).  The links cross PCIe once each way. */
int gfix_coulomb_driver(double *links, const size_t dims[4], const gfix_params *p,
                        gfix_result *r, double *obs_in, double *diag_in,
                        double *obs, double *diag);

/* As gfix_landau, but `d_links` is a device pointer to the same layout
 * (links already resident in HBM); nothing crosses PCIe but scalars. */
int gfix_landau_device(double *d_links, const size_t dims[4],
                       const gfix_params *p, gfix_result *r);

/* Coulomb FA gauge fixing of host links in place: every time slice solved
 * as an independent 3D problem in one batched launch sequence, then the
 * slice transforms (no final reunitarisation; gfix_reunit does that).
 * slice_theta / slice_iters (length Lt, may be NULL) receive per-slice
 * results; traj_theta records the accelerated theta of every slice at every
 * FFT round, slice-major with stride traj_cap / Lt. */
int gfix_coulomb(double *links, const size_t dims[4], const gfix_params *p,
                 gfix_result *r, double *slice_theta, size_t *slice_iters);

int gfix_coulomb_device(double *d_links, const size_t dims[4],
                        const gfix_params *p, gfix_result *r,
                        double *slice_theta, size_t *slice_iters);

/* Batches: many configurations, of any shapes, Landau-fixed together (no
 * counterpart in GLU, which fixes one configuration per call).  Every
 * configuration keeps its own device workspace; one CUDA graph launch
 * advances all unfinished ones concurrently, and a converged configuration
 * drops out (its kernels turn into no-ops, the graph is rebuilt without it
 * as the live set shrinks).  Each configuration's result equals that of
 * gfix_landau with the same parameters (trajectories are not recorded).
 *
 *   gfix_batch *b = gfix_batch_create(&p);
 *   gfix_batch_add(b, links_a, dims_a);         // index 0
 *   gfix_batch_add(b, links_b, dims_b);         // index 1
 *   gfix_batch_run(b);                           // links fixed in place
 *   gfix_batch_result(b, 0, &r);
 *   gfix_batch_destroy(b);
 *
 * add returns the configuration's index or -1; the links must stay valid
 * until the run returns.  gfix_batch_add_device takes links in HBM. */
typedef struct gfix_batch gfix_batch;
gfix_batch *gfix_batch_create(const gfix_params *p);
int gfix_batch_add(gfix_batch *b, double *links, const size_t dims[4]);
int gfix_batch_add_device(gfix_batch *b, double *d_links, const size_t dims[4]);
int gfix_batch_run(gfix_batch *b);
int gfix_batch_result(const gfix_batch *b, int i, gfix_result *r);
void gfix_batch_destroy(gfix_batch *b);

/* Coulomb fixing of one rank's block of time slices of a larger lattice
 * (slices are independent problems; GLU's Coulomb_FA, CFACG.c:531-636,
 * fixes them one after the other).  d_links: the block's links in HBM,
 * double[V][4][9][2] for dims = {Lx, Ly, Lz, T_block >= 2}.  Solves every
 * slice, applies the slice transforms except to the temporal links of the
 * block's last slice, and writes the gauge fields of the block's first and
 * last slices to d_g_first / d_g_last (double[9][Lx Ly Lz][2] in HBM).
 * gfix_coulomb_slices_finish then transforms those last temporal links with
 * d_g_last and the following block's d_g_first (d_g_next, from the rank
 * that owns the following slice).  Over all blocks this equals gfix_coulomb
 * on the whole lattice, bit for bit. */
int gfix_coulomb_slices(double *d_links, const size_t dims[4],
                        const gfix_params *p, gfix_result *r,
                        double *slice_theta, size_t *slice_iters,
                        double *d_g_first, double *d_g_last);
int gfix_coulomb_slices_finish(double *d_links, const size_t dims[4],
                               const double *d_g_last, const double *d_g_next);

/* Observables on host links: theta_test_lin (src/Gfix/gftests.c:214-250),
 * gauge functional (gftests.c:132-147), average plaquette
 * (src/Field/plaqs_links.c:243-265).  out[0..2] in that order. */
int gfix_observables(const double *links, const size_t dims[4], double *out);

/* GLU's post-fix link diagnostics on host links (output_fixing_info,
 * src/Gfix/Landau.c:42-66; all_links in Coulomb, Coulomb.c:37-41):
 * out[0] spatial and out[1] temporal average Re tr / NC (all_links,
 * src/Field/plaqs_links.c:399-420), out[2] average Re tr / NC of all links
 * and out[3] the largest Re tr / NC (indivlinks, plaqs_links.c:424-446),
 * out[4] and out[5] the temporal constancy, linear and logarithmic
 * definitions (const_time, src/Gfix/gftests.c:35-129).  out holds 6. */
int gfix_link_diagnostics(const double *links, const size_t dims[4],
                          double *out);

/* GLU's gauge-fixing accuracy report (gf_check, src/Wrappers/OBS_wrap.c:
 * 93-126) of host links: out[0] theta_test_lin and out[1] its largest local
 * value over the four directions (Landau; src/Gfix/gftests.c:214-250),
 * out[2], out[3] the same by the logarithmic definition (theta_test_log,
 * gftests.c:253-290), out[4], out[5] the temporal constancy (const_time,
 * linear and logarithmic), out[6..9] as out[0..3] over the three spatial
 * directions (Coulomb).  out holds 10.  A link whose three eigenvalue
 * phases are equal (the identity) contributes a zero logarithm. */
int gfix_gf_check(const double *links, const size_t dims[4], double *out);

/* Reunitarise every link (GLU's latt_reunitU, src/Geometry/random_config.c:
 * 42-57) on the GPU, host links in place. */
int gfix_reunit(double *links, const size_t dims[4]);

/* In place: fields (4 packed fields of vol complex numbers each, double[4]
 * [vol][2]) <- IDFT(psq * DFT(fields)) over ndim = 4 (dims[0..3]) or 3
 * (one slice, dims[0..2]); psq = MAX / p^2 as GLU builds it. */
int gfix_fourier_accelerate(double *fields, const size_t dims[4], int ndim);

/* Measurement aid: run `iters` Landau CG iterations from the device links
 * `d_links` (not modified) with CUDA events between the kernel launches.
 * ms[k] = mean duration of one launch of kernel k, bytes[k] = algorithmic
 * HBM bytes of one launch, for k = 0 derivative+theta, 1 xy FFT forward,
 * 2 zt FFT with psq, 3 xy FFT inverse + PR sums, 4 direction + line-search
 * probes, 5 link update, 6 the scalar-control launches of one iteration.
 * precision GFIX_MIXED profiles the FP32 kernels, GFIX_PROFILE_POLISH those
 * of a mixed solve's FP64-link phase. */
int gfix_profile_landau(const double *d_links, const size_t dims[4],
                        const gfix_params *p, int iters, double *ms,
                        double *bytes);

/* Measurement aid for Coulomb: `iters` steps of every slice from the device
 * links `d_links` (not modified), accuracy forced to 0 so no slice stops,
 * with CUDA events between the launches.  ms[k] / bytes[k] as for
 * gfix_profile_landau, for k = 0 derivative, 1 xy FFT forward, 2 z FFT with
 * psq, 3 xy FFT inverse + the per-slice sums, 4 direction + line-search
 * probes, 5 update of the slice gauge fields, 6 the scalar, housekeeping and
 * parity launches of one step.  precision GFIX_MIXED profiles the FP32
 * kernels. */
int gfix_profile_coulomb(const double *d_links, const size_t dims[4],
                         const gfix_params *p, int iters, double *ms,
                         double *bytes);

/* theta_test_lin (src/Gfix/gftests.c:214-250) and the gauge functional
 * (gftests.c:132-147) of the device links d_links (double[V][4][9][2] in
 * HBM), written to the device array d_out[0..1].  No counterpart in the
 * reference: it serves callers that cannot allocate device memory when they
 * call in -- codes that give all of HBM to their own arena allocator, and
 * stream-ordered pipelines in which cudaMalloc/cudaFree would synchronise
 * the device.  It allocates nothing: its scratch is a fixed 1 MiB device
 * array inside the library, so lattices above 16,777,216 sites are rejected.
 * Calls that overlap on the GPU race on that array.  The first call on a
 * device looks the array up; make it before any stream capture.  stream is
 * a cudaStream_t (NULL: the legacy default stream); both kernels are
 * launched on it and the call returns without waiting for them, so d_out
 * is ready once the stream's work up to this call has completed.  Returns
 * 0, or -1 with the reason in gfix_noalloc_error() (thread-local). */
int gfix_theta_functional_noalloc(const double *d_links, const size_t dims[4],
                                  double *d_out, void *stream);
const char *gfix_noalloc_error(void);

/* FFT plans.  0 (default): a fixed plan per lattice shape -- compile-time
 * passes where the extents have one, largest radices first -- so repeated
 * runs are bit-identical.  1: at the first use of a shape every available
 * xy and z(,t) pass is timed once (compile-time or generic, each radix order
 * of the generic pass, every zt tile width dividing Lx) and the fastest is
 * kept for the process; plans differ in rounding only.  The environment
 * variable GLU_GFIX_FFT_TUNE=1 sets 1 at load.  Switching drops the cached
 * workspaces. */
void gfix_fft_tuning(int on);

/* The plan of a shape (building its workspace): plan[0] = xy pass (-1
 * compile-time, else the generic pass's radix order), plan[1] = zt tile
 * width, plan[2] = zt pass (-1 compile-time, else radix order); ms[0..1]
 * (may be NULL) the measured times of the tuned xy / zt pass (0 untuned).
 * coulomb: 1 for the Coulomb workspace (3D FFT per slice);
 * precision: GFIX_MIXED reports the FP32 workspace. */
int gfix_fft_plan(const size_t dims[4], int coulomb, int precision, int *plan,
                  float *ms);

/* NERSC configuration payloads on the GPU (GLU's I/O layer,
 * src/IO/readers.c:169-310, src/IO/writers.c): the binary part of a NERSC
 * file -- per site (x fastest), per direction, nreal = 12 (4D_SU3_GAUGE, the
 * top two rows; the third is completed as conj(row0 x row1),
 * readers.c:50-58) or 18 (4D_SU3_GAUGE_3x3) reals of bytes_per_real = 8
 * (IEEE64) or 4 (IEEE32), big-endian when big_endian != 0 -- to GLU's
 * double[V][4][9][2] links and back.  *checksum (may be NULL) receives the
 * NERSC checksum: the 32-bit wrapping sum over the stored numbers, in host
 * byte order, of their 32-bit words (readers.c:279-293).  Header lines are
 * the caller's (glu_b200/nersc.py parses and writes them).  Host pointers;
 * returns 0 or -1 with the reason in gfix_nersc_error(). */
int gfix_nersc_decode(const void *payload, const size_t dims[4], int nreal,
                      int bytes_per_real, int big_endian, double *links,
                      uint32_t *checksum);
int gfix_nersc_encode(const double *links, const size_t dims[4], int nreal,
                      int bytes_per_real, int big_endian, void *payload,
                      uint32_t *checksum);
const char *gfix_nersc_error(void);

/* SCIDAC / ILDG checksums of a payload of nsites records of site_bytes
 * bytes each, as stored (src/IO/writers.c:210-224, readers.c:256-263): per
 * site the CRC-32 of its bytes, rotated left by site % 29 (suma) and by
 * site % 31 (sumb), XORed over the sites.  The ILDG payload itself decodes
 * with gfix_nersc_decode (18 reals, big-endian).  Host pointers. */
int gfix_scidac_checksum(const void *payload, size_t site_bytes, size_t nsites,
                         uint32_t *suma, uint32_t *sumb);

/* Momentum-space gluon measurements (GLU's cuts_struct, src/Cuts/cuts.c:
 * 110-184, as cuts_wrap_struct calls it for CUTTYPE = GLUON_PROPS,
 * EXCEPTIONAL and FIELDS, src/Wrappers/CUT_wrap.c:57-63).  The fields of
 * GLU's struct cut_info (src/Headers/GLU_types.h:94-103) these modes read;
 * enum values are GLU's (src/Headers/GLU_enum.h:161-195). */
enum {
  GFIX_CUT_EXCEPTIONAL = 0,    /* MOMgg g2, g3 (src/Cuts/MOMgg.c) */
  GFIX_CUT_NONEXCEPTIONAL = 1, /* not provided */
  GFIX_CUT_FIELDS = 2,         /* the fields at the kept momenta */
  GFIX_CUT_GLUON_PROPS = 6     /* transverse / longitudinal (glueprop.c) */
};
enum {
  GFIX_CUT_HYPERCUBIC = 0,
  GFIX_CUT_PSQ = 1, /* SPHERICAL_CUT in the input file */
  GFIX_CUT_CYLINDER = 2,
  GFIX_CUT_CONICAL = 3
};
enum { GFIX_FIELD_LINEAR = 0, GFIX_FIELD_LOG = 1 };

typedef struct gfix_cut_info {
  int dir;          /* GFIX_CUT_GLUON_PROPS, _EXCEPTIONAL or _FIELDS */
  int type;         /* momentum cut, GFIX_CUT_HYPERCUBIC .. _CONICAL */
  size_t max_mom;   /* MAXMOM: largest (n_mu small/L_mu)^2 kept */
  int definition;   /* GFIX_FIELD_LINEAR (Hermitian projection) or
                       GFIX_FIELD_LOG (exact logarithm) */
  size_t angle;     /* ANGLE of the conical cut, degrees */
  double cyl_width; /* CYL_WIDTH in units of 2 pi / min(L) */
} gfix_cut_info;

/* compute_veclist (src/Cuts/cut_routines.c:459-631) in momentum space: the
 * number of kept momenta (or -1); with mom, up to cap momenta as 4 ints
 * each in GLU's order (lexicographic in the -pi..pi zone, x fastest).
 * Host-only: needs no GPU. */
long gfix_cut_veclist(const size_t dims[4], const gfix_cut_info *ci,
                      int32_t *mom, size_t cap);

/* the measurement of cuts_struct without its file: links are GLU's
 * double[V][4][9][2] (host, or device for _device); nmom must be the count
 * of gfix_cut_veclist.  GLUON_PROPS: out0 = transverse G(p^2), out1 =
 * longitudinal F(p^2) (glueprop.c:89-146); EXCEPTIONAL: out0 = g2, out1 =
 * g3 (MOMgg.c:160-211); FIELDS: out0 = nmom * 4 * 9 complex fields
 * (interleaved re, im) times e^{i p_mu/2}, out1 unused.  pspace_err
 * (may be NULL) receives the p-space gauge error GLU prints
 * (src/Cuts/pspace_landau.c:78-80). */
int gfix_cuts_measure(const double *links, const size_t dims[4],
                      const gfix_cut_info *ci, size_t nmom, double *out0,
                      double *out1, double *pspace_err);
int gfix_cuts_measure_device(const double *d_links, const size_t dims[4],
                             const gfix_cut_info *ci, size_t nmom,
                             double *out0, double *out1, double *pspace_err);

/* cuts_struct itself: measures and writes GLU's output file (big-endian,
 * src/Cuts/cut_output.c:250-410), named as output_str_struct does
 * (cut_output.c:121-242) after the prefix `where` (GLU's default build
 * uses "./"); flow is the configuration number in the name.  The path is
 * copied to path_out (may be NULL). */
int gfix_cuts_write(const double *links, const size_t dims[4],
                    const gfix_cut_info *ci, const char *where, size_t flow,
                    double *pspace_err, char *path_out, size_t path_cap);

/* per-kernel CUDA-event times (ms, mean of reps after one warm-up) of the
 * measurement on device links: [0] Lie fields + x,y transforms, [1] z,t
 * transforms, [2] gather + contraction */
int gfix_profile_cuts(const double *d_links, const size_t dims[4],
                      const gfix_cut_info *ci, int reps, float ms[3]);

const char *gfix_cuts_error(void);
void gfix_cuts_release(void);

/* Quenched SU(3) configurations by heatbath and over-relaxation (GLU's
 * hb_update, src/Update/KPHB.c:123-257, MODE = HEATBATH): each of
 * `iterations` steps is one heatbath sweep (hb_lattice, src/Update/hb.c:
 * 146-194: Kennedy-Pendleton per SU(2) subgroup, links reunitarised) and
 * n_or over-relaxation sweeps (OR_lattice, src/Update/relax.c:83-114), in
 * GLU's order (per direction, per draughtboard colour).  beta is the Wilson
 * coupling; random numbers are Philox4x32-10 keyed by `seed`, the counter
 * holding the step number first_iteration + i, so a run continued from
 * (seed, first_iteration) equals the uninterrupted one.  plaquettes (may be
 * NULL) receives the average plaquette after every step.  Even extents
 * only.  Links as everywhere: double[V][4][9][2], host or device. */
int gfix_heatbath(double *links, const size_t dims[4], double beta,
                  size_t iterations, size_t n_or, uint64_t seed,
                  uint64_t first_iteration, double *plaquettes);
int gfix_heatbath_device(double *d_links, const size_t dims[4], double beta,
                         size_t iterations, size_t n_or, uint64_t seed,
                         uint64_t first_iteration, double *plaquettes);

/* `sweeps` over-relaxation sweeps alone (deterministic: no random numbers) */
int gfix_overrelax(double *links, const size_t dims[4], size_t sweeps);

/* the generator's block function: Philox4x32-10 of counter ctr under key
 * (host only) */
void gfix_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                        uint32_t out[4]);

const char *gfix_update_error(void);
void gfix_update_release(void);

/* message of the last failed call (thread-local, never NULL) */
const char *gfix_last_error(void);

/* free the cached device workspaces */
void gfix_release(void);

/* number of kernels launched by this library since load (all devices) */
unsigned long long gfix_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* GLU_B200_GFIX_H */
