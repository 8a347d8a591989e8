/*
 * CPU oracle for the ARMA wavy-surface hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C++17 with no third-party dependencies,
 * the reference implementation's algorithm for every row of the hot path
 * (analytic ACF, block-Toeplitz Yule-Walker system, white-noise variance,
 * dcmt Mersenne Twister draws, libstdc++ normal white noise, the causal 3-D
 * AR filter, the OpenMP block wavefront, variance renormalisation, the NIT
 * bisection and the linear velocity-potential solver).  Each function cites
 * the reference file:line it follows (paths relative to the reference
 * project root).
 *
 * It is a checker.  Only the test-suite, the smoke check and the benchmark's
 * CPU-baseline leg may load it; the product library never links or calls it.
 *
 * Parity status:
 *   - MT recurrence/tempering/seeding: pinned against libstdc++ std::mt19937
 *     (the standard MT19937 parameter set expressed as a dcmt mt_struct) and
 *     against the C++ standard's 10000th-draw requirement.  Byte-level
 *     equality with libdcmt's own output for dcmt-created parameter sets is
 *     unpinned (libdcmt is absent from this build environment).
 *   - Normal white noise: libstdc++ std::normal_distribution is called
 *     directly (pinned by construction).
 *   - dsysv / Owen T / skew-normal CDF / config grammar: pinned against the
 *     reference test-suite's known answers (tests/golden).
 *   - AR filter, renormalisation, NIT realisation and the linear solver have
 *     no reference golden vectors: parity is pinned by restatement only.
 */
#ifndef ARMA_ORACLE_H
#define ARMA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* dcmt mt_struct field order (reference src/parallel_mt.hh:109-123). */
typedef struct {
	uint32_t aaa;
	int32_t mm, nn, rr, ww;
	uint32_t wmask, umask, lmask;
	int32_t shift0, shift1, shiftB, shiftC;
	uint32_t maskB, maskC;
	int32_t i;
} orc_mt_params;

/* ---- A1: analytic ACF (src/acf.hh:18-62) ---- */
void orc_acf_standing(double amplitude, double velocity, const double alpha[3],
                      const double beta[2], const double delta[3],
                      int nt, int nx, int ny, double* out);
void orc_acf_propagating(double amplitude, double velocity, const double alpha[3],
                         const double beta[2], const double delta[3],
                         int nt, int nx, int ny, double* out);

/* ---- A2: block-Toeplitz auto-covariance matrix (src/generator/voodoo.cc:58-104) ---- */
void orc_ac_matrix(const double* acf, int at, int ax, int ay,
                   int pt, int px, int py, double* out /* P*P */);

/* ---- linalg (src/linalg.cc:22-35): symmetric indefinite solve ---- */
int orc_sysv_upper(int n, double* a /* n*n row-major, destroyed */, double* b);
int orc_cholesky_solve(int n, double* a /* n*n row-major, destroyed */, double* b);

/* ---- A3 + A4: Gauss-elimination YW fit (src/generator/ar_model.cc:97-135, 55-61)
 * method 0 = Bunch-Kaufman (reference dsysv), 1 = Cholesky LL^T. ---- */
int orc_ar_fit_gauss(const double* acf, int at, int ax, int ay,
                     int pt, int px, int py, int method,
                     double* phi /* pt*px*py */, double* var_wn);
double orc_white_noise_variance(const double* acf, int at, int ax, int ay,
                                const double* phi, int pt, int px, int py);

/* ---- A6: dcmt Mersenne Twister (src/parallel_mt.hh:61-275, src/parallel_mt.cc:28-59) ---- */
void orc_mt_sgenrand(const orc_mt_params* p, uint32_t seed, uint32_t* state);
/* Draw n words starting from a freshly seeded state. */
void orc_mt_genrand(const orc_mt_params* p, uint32_t seed, size_t n, uint32_t* out);
/* Standard MT19937 parameter set in dcmt form. */
void orc_mt19937_params(orc_mt_params* p);
/* std::mt19937 draws for pinning the restatement. */
void orc_std_mt19937(uint32_t seed, size_t n, uint32_t* out);
/* mt.dat IO: raw x86-64 mt_struct (72 bytes) followed by nn state words. */
int orc_mt_file_count(const char* path);
int orc_mt_file_read(const char* path, int index, orc_mt_params* p);
int orc_mt_file_write(const char* path, const orc_mt_params* p, int n,
                      const uint32_t* states /* concatenated nn words each */);

/* ---- A7: white noise (src/white_noise.hh:23-58) ---- */
void orc_white_noise(const orc_mt_params* p, uint32_t seed, double stddev,
                     size_t n, double* out);
/* Number of MT words consumed to produce n normals (for sizing). */
size_t orc_white_noise_words(const orc_mt_params* p, uint32_t seed, size_t n);

/* ---- A8: causal AR filter, in place (src/generator/ar_model_surf.cc:5-36) ---- */
void orc_ar_filter(double* zeta, int nt, int nx, int ny,
                   const double* phi, int pt, int px, int py);
void orc_ar_filter_f32(float* zeta, int nt, int nx, int ny,
                       const float* phi, int pt, int px, int py);

/* ---- A9: OpenMP block wavefront (src/generator/ar_model_parallel.cc:76-201).
 * with_noise=1 fills each partition from a per-thread MT as the reference
 * does (non-deterministic partition->thread mapping); with_noise=0 filters an
 * already-filled zeta and is bit-identical to orc_ar_filter. ---- */
int orc_ar_generate_omp(double* zeta, int nt, int nx, int ny,
                        const double* phi, int pt, int px, int py,
                        int with_noise, const orc_mt_params* params, int nparams,
                        const uint32_t* seeds, double stddev, int nthreads,
                        const int partition[3]);
void orc_partition_shape(const int grid[3], const int order[3], int parallelism,
                         const int user[3], int out[3]);

/* ---- A10: variance renormalisation (src/generator/basic_arma_model.cc:102-106) ---- */
double orc_variance_renorm(double* zeta, int nt, int nx, int ny, double acf0);
double orc_variance_unbiased(const double* x, size_t n);

/* ---- A11: NIT (src/nonlinear/transforms.hh:58-75, src/linalg.hh:199-268) ---- */
double orc_gaussian_cdf(double x, double mean, double sigma);
double orc_owen_t(double h, double a);
double orc_skew_normal_cdf(double x, double mean, double sigma, double alpha);
double orc_gram_charlier_cdf(double x, double skewness, double kurtosis);
/* kind 0 = Gram-Charlier(p0=skewness, p1=kurtosis), 1 = skew normal(p0=mean,
 * p1=stdev, p2=alpha). */
void orc_nit_transform(double* data, size_t n, double stdev, int kind,
                       const double params[3], double a, double b, double eps,
                       int max_iter, int nthreads);

/* ---- V1-V5: linear velocity-potential solver (src/velocity/basic_solver.cc, linear_solver.cc) ---- */
void orc_derivative_t(const double* zeta, int nt, int nx, int ny, double dt,
                      int idx_t, double* out);
void orc_factor_waves(const double* slice, int nx, int ny, int t, double dt,
                      double out_min[2], double out_max[2]);
void orc_window_function(int nx, int ny, double wnmax_x, double wnmax_y,
                         double z, double depth, double* out);
void orc_fft2(double* re, double* im, int nx, int ny, int sign);
void orc_velocity_linear(const double* zeta, int nt, int nx, int ny,
                         const double delta[3], double depth,
                         const double* z, int nz, const int* t_idx, int ntd,
                         double* out /* ntd*nz*nx*ny */, int nthreads);
void orc_velocity_solve(int mode, const double* zeta, int nt, int nx, int ny,
                        const double delta[3], double depth, const double* zs, int nz,
                        const int* t_idx, int ntd, double* out, int nthreads);

/* ---- O1: output layout (src/arma_driver.cc:29-69) ---- */
int orc_write_zeta_bin(const char* path, const double* zeta, size_t n);
int orc_write_zeta_csv(const char* path, const double* zeta, int nt, int nx,
                       int ny, const double delta[3]);

/* ---- M: moving-average model (ma.cc) ---- */
/* fixed-point MA fit: 0 ok, 1 bad order, 2 non-finite, 3 variance <= 1e-6 */
int orc_ma_fit(const double* acf, int at, int ax, int ay, int pt, int px, int py,
               double* theta, double* var_wn, int* iterations);
/* direct MA sum zeta = eps - sum_{m != 0} theta(m) eps(n - m) */
void orc_ma_filter(const double* theta, int pt, int px, int py, const double* eps, int nt,
                   int nx, int ny, double* zeta);

#ifdef __cplusplus
}
#endif

#endif
