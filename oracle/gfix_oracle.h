/*
 * CPU oracle: a plain-C restatement of GLU's Fourier-accelerated Landau and
 * Coulomb gauge fixing (FACG / FASD), SU(3), ND = 4, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (glu_b200/) never links, loads or
 * calls this code; the tests, the smoke check and the CPU-baseline leg of
 * the benchmark use it as the checker.
 *
 * Link layout: double[V][4][9][2] (site x fastest, mu, row-major 3x3
 * complex as (re,im)), GLU's in-memory order of lat[i].O[mu][a*3+b].
 * Field layout: double[4][V][2] (the four packed su(3) fields of GLU's
 * SU(3) trick, src/Gfix/FACG.c:54-60).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef GLU_B200_GFIX_ORACLE_H
#define GLU_B200_GFIX_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GLU's non-convergence sentinel (src/Gfix/FACG.c:381) */
#define ORC_SENTINEL ((size_t)123456789)

/* Landau FA gauge fixing in place.  algo 0 = FACG (src/Gfix/FACG.c:341),
 * 1 = FASD (src/Gfix/FACG.c:395).  sd_fixed_step != 0 reproduces a GLU
 * build with GLU_GFIX_SD (fixed step gf_alpha instead of the line search
 * in the steepest-descent step, src/Gfix/FACG.c:192-196).  Returns the
 * reference's iteration count (or sentinel); *theta receives the final
 * in-loop theta.  Trajectories (theta and functional evaluated on the links
 * at every derivative evaluation, SD start included) go to traj_* when
 * traj_cap > 0. */
size_t orc_landau_fa(double *links, const size_t dims[4], double gf_alpha,
                     double acc, size_t max_iters, int algo,
                     int sd_fixed_step, double *theta, double *traj_theta,
                     double *traj_func, size_t traj_cap, size_t *traj_len);

/* Coulomb FA gauge fixing in place (src/Gfix/CFACG.c:531), all slices in
 * GLU's order, including the slice transforms of the links; no final
 * reunitarisation (see orc_reunit_links).  facg 1 = FACG, 0 = FASD.
 * slice_theta/slice_iters (length dims[3]) receive each slice's final
 * theta and iteration total; traj_* the accelerated theta of every FFT
 * round, slices concatenated in order; *restarts the random restarts. */
size_t orc_coulomb_fa(double *links, const size_t dims[4], double gf_alpha,
                      double acc, size_t max_iters, int facg,
                      int sd_fixed_step, double *slice_theta,
                      size_t *slice_iters, double *traj_theta,
                      size_t traj_cap, size_t *traj_len, size_t *restarts);

/* single pieces of the path, for kernel-level checks */
double orc_theta_test_lin(const double *links, const size_t dims[4]);
double orc_gauge_functional(const double *links, const size_t dims[4]);
double orc_plaquette(const double *links, const size_t dims[4]);
void orc_reunit_links(double *links, size_t nlinks);
/* packed derivative fields[4][V] and the in-loop theta (FA_deriv) */
double orc_derivative(const double *links, const size_t dims[4],
                      double *fields);
/* in place: fields <- IDFT(psq * DFT(fields)) over ndim = 4 (Landau) or 3
 * (Coulomb, one slice of dims[0..2]) */
void orc_fourier_accelerate(double *fields, const size_t dims[4], int ndim);
/* the p^2 table psq[i] = (4 ndim / vol) / p^2(i) */
void orc_psq(double *psq, const size_t dims[4], int ndim);
/* plain multi-dimensional DFT (row-major over n[0..rank-1]) */
void orc_dft(double *data, int rank, const int *n, int sign);
/* PR sums: out[0] = insum, out[1] = sum_conj (src/Gfix/FACG.c:99-145) */
void orc_sum_pr(const double *in, const double *in_old, size_t V,
                double *out);
/* Landau line-search probe values val[3] for direction sn
 * (src/Gfix/line_search.c:274-341) and the chosen step */
double orc_line_search_probes(const double *links, const size_t dims[4],
                              const double *sn, double *val);
/* U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag, g = reunit(1 + alpha A)
 * (src/Gfix/line_search.c:60-97) */
void orc_link_update(double *links, const size_t dims[4], const double *sn,
                     double alpha);
/* g = reunit(1 + alpha A(in, i)) as 3x3 (src/Gfix/CG.c:46-100) */
void orc_gauge_matrix(const double *fields, size_t V, size_t i, double alpha,
                      double *g);
/* in-place column Gram-Schmidt of a 3x3 (src/Matrix_Ops/gramschmidt_SSE.c) */
void orc_gram_reunit(double *u);
/* approx_minimum (src/Gfix/line_search.c:38-57) */
double orc_approx_minimum(const double *alphas, const double *vals);

#ifdef __cplusplus
}
#endif

#endif
