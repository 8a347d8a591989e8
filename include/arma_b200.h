/*
 * arma_b200 — C ABI of the B200 implementation of the ARMA wavy-surface hot
 * path: Yule-Walker fit, dcmt Mersenne Twister white noise, the causal 3-D AR
 * filter, variance renormalisation, the nonlinear inertialess transform and
 * the linear velocity-potential solver.
 *
 * Conventions
 *   - Every entry point returns an int status: ARMA_OK (0) or a negative
 *     ARMA_E* code.  arma_last_error() returns the calling thread's message.
 *     No C++ exception crosses this boundary.
 *   - Arrays are C order with t slowest: zeta is (nt, nx, ny), phi is
 *     (pt, px, py), velocity potentials are (nt_dom, nz, nx, ny), exactly the
 *     blitz layouts of the reference (src/arma_driver.hh:56-57).
 *   - Pointers named d_* are device pointers on the context's device; all
 *     other pointers are host pointers.  Device work is enqueued on the
 *     context's stream (arma_ctx_set_stream); calls that return host results
 *     synchronise that stream.
 *   - A context is used by one host thread at a time.
 *
 * The reference has no C ABI; its operator API is the C++ generator/solver
 * registry (src/arma_driver.hh:124-134) with the virtual interfaces cited on
 * each entry point below.
 */
#ifndef ARMA_B200_H
#define ARMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARMA_B200_VERSION 100

enum {
	ARMA_OK = 0,
	ARMA_EINVAL = -1,     /* bad argument (std::invalid_argument in the reference) */
	ARMA_ECUDA = -2,      /* CUDA runtime error */
	ARMA_ENOMEM = -3,     /* device allocation failed */
	ARMA_ETIMEDOUT = -4,  /* a bounded device-side wait gave up */
	ARMA_EIO = -5,        /* file missing or malformed (std::runtime_error) */
	ARMA_EPRNG = -6,      /* too few MT parameter sets (PRNG_error, src/errors.hh:10-33) */
	ARMA_ENUMERIC = -7,   /* singular YW system or negative white-noise variance */
	ARMA_ENOTSUP = -8     /* registered but not built in this library */
};

typedef enum { ARMA_FP64 = 0, ARMA_FP32C = 1 } arma_precision;
typedef enum { ARMA_ACF_STANDING = 0, ARMA_ACF_PROPAGATING = 1 } arma_acf_kind;
typedef enum {
	ARMA_FIT_BUNCH_KAUFMAN = 0, /* reference dsysv semantics, per-axis |lag| matrix */
	ARMA_FIT_CHOLESKY = 1       /* LL^T, per-axis |lag| matrix */
} arma_fit_method;
typedef enum { ARMA_NIT_GRAM_CHARLIER = 0, ARMA_NIT_SKEW_NORMAL = 1 } arma_nit_dist;
typedef enum { ARMA_NIT_BISECTION = 0, ARMA_NIT_LUT = 1 } arma_nit_method;

/* One dcmt parameter set: the reference's mt_struct fields in order
 * (src/parallel_mt.hh:109-123; on disk in mt.dat as the raw x86-64 struct,
 * 72 bytes, followed by nn state words). */
typedef struct {
	uint32_t aaa;
	int32_t mm, nn, rr, ww;
	uint32_t wmask, umask, lmask;
	int32_t shift0, shift1, shiftB, shiftC;
	uint32_t maskB, maskC;
	int32_t i;
} arma_mt_params;

typedef struct arma_ctx arma_ctx;

/* ---------------------------------------------------------------- context */
int arma_version(void);
int arma_last_error(char* buf, size_t len);
int arma_ctx_create(int device, arma_ctx** out);
int arma_ctx_destroy(arma_ctx* ctx);
int arma_ctx_set_stream(arma_ctx* ctx, void* cuda_stream);
int arma_ctx_synchronize(arma_ctx* ctx);
/* Kernel launches issued through this context since creation (counter). */
int arma_ctx_launch_count(arma_ctx* ctx, uint64_t* count);
/* Bytes the context's calls have copied host->device and device->host since
 * creation (counters): inputs, descriptors, coefficient tables, results. */
int arma_ctx_transfer_bytes(arma_ctx* ctx, uint64_t* h2d, uint64_t* d2h);
/* Per-kernel-class device timing: when enabled, CUDA events are recorded on
 * the context's stream around each launch of the named classes ("mt",
 * "noise", "ar64", "ar32c", "renorm", "nit", "velocity").  arma_ctx_profile
 * synchronises and returns the accumulated milliseconds and launch count of
 * one class (zeros if none ran); arma_ctx_profile_reset clears them. */
int arma_ctx_set_profiling(arma_ctx* ctx, int enabled);
int arma_ctx_profile(arma_ctx* ctx, const char* name, double* ms, uint64_t* launches);
int arma_ctx_profile_reset(arma_ctx* ctx);
/* Settings of the batched calls that change their speed but never their
 * results (no counterpart in the reference):
 *   mt_log2_segment  the dcmt stream of a surface is cut into segments of
 *                    2^v words generated by one CTA each, v in [16, 22]
 *                    (default 20); shorter segments give more CTAs and more
 *                    jump-ahead work;
 *   ar_ctas_per_sm   CTAs of the persistent FP32 filter launch per SM, 0 =
 *                    as many as fit (default);
 *   host_groups      arma_batch_generate_host (FP32) splits the batch, in
 *                    order of the filter's dependency chain, into this many
 *                    groups, 1..16 (default 16), computed on two alternating
 *                    streams, whose device->host copies overlap the later
 *                    groups' computation;
 *   host_first       share of the work in the first group, (0, 1) (default
 *                    0.06); the other groups share the rest equally.
 * arma_autotune (after the batch calls below) picks them for a batch by
 * timing. */
typedef struct {
	int mt_log2_segment;
	int ar_ctas_per_sm;
	int host_groups;
	double host_first;
} arma_tuning;
int arma_ctx_get_tuning(arma_ctx* ctx, arma_tuning* out);
int arma_ctx_set_tuning(arma_ctx* ctx, const arma_tuning* t);
/* Multiplier (> 0, default 1) of the polar-attempt estimate (expected count
 * plus 8 sigma) with which the batched generation calls (arma_batch_generate,
 * arma_batch_generate_host, arma_ma_generate) draw each surface's dcmt words.
 * No counterpart in the reference, which draws one word at a time.  A
 * surface whose noise runs short is generated again on its own, so the
 * results do not depend on it; values below 1 make that path likely. */
int arma_ctx_set_noise_margin(arma_ctx* ctx, double margin);

/* ------------------------------------------------- A6: dcmt parameter sets */
/* Replaces read_parallel_mt_config / read_parallel_mts
 * (src/parallel_mt.hh:153-168, src/parallel_mt.cc:28-59). */
int arma_mt_file_count(const char* path, int* count);
int arma_mt_file_read(const char* path, int index, arma_mt_params* out);
/* Writes n sets, each followed by nn state words seeded with 0 (the
 * reference's arma-dcmt writes its creator state; seeding replaces it). */
int arma_mt_file_write(const char* path, const arma_mt_params* sets, int n);
/* The standard MT19937 parameter set in dcmt form. */
int arma_mt19937_params(arma_mt_params* out);
/* Creates the dcmt parameter set of generator `id` (0 <= id < 65536) of period
 * 2^p - 1, w = 32: replaces get_mt_parameter_id_st(32, p, id, seed), which the
 * reference's parallel_mt_seq calls (src/parallel_mt.hh:199-203) for
 * arma-dcmt (src/dcmt.cc:15-33; p = 521 there).  p must be a Mersenne
 * exponent (521, 607, 1279, 2203, 2281, 3217, 4253, 4423, 9689, 9941, 11213,
 * 19937, 21701, 23209, 44497).  The result depends only on (p, id, seed).
 * The id sits in the low 16 bits of aaa; when none of the 2^15 twist vectors
 * of that id gives a primitive characteristic polynomial the call fails with
 * ARMA_ENUMERIC (the reference then throws "bad MT"). */
int arma_mt_create(int w, int p, int id, uint32_t seed, arma_mt_params* out);
/* *primitive = 1 when the set's characteristic polynomial is primitive
 * (period 2^p - 1 with p = 32 nn - rr a Mersenne exponent), else 0. */
int arma_mt_is_primitive(const arma_mt_params* p, int* primitive);
/* k_out[v-1] = k(v), v = 1..vmax (vmax <= 32): the dimension of
 * equidistribution of the top v bits of the tempered output (-1 where the
 * lattice reduction did not close). */
int arma_mt_equidistribution(const arma_mt_params* p, int vmax, int* k_out);
/* n tempered words of the stream seeded with `seed` (sgenrand_mt then
 * genrand_mt, src/parallel_mt.hh:236,259), starting at word `offset`. */
int arma_mt_genrand(arma_ctx* ctx, const arma_mt_params* p, uint32_t seed,
                    uint64_t offset, size_t n, uint32_t* d_out);

/* ------------------------------------------------------ A1-A5: model fit */
/* Circular auto-covariance of an n0 x n1 x n2 FP64 array (row-major, t
 * slowest): out(i,j,k) = sum w(i1,j1,k1) w((i+i1)%n0,(j+j1)%n1,(k+k1)%n2) / n,
 * computed as Re IFFT(|FFT(w)|^2) / n / n in FP64 on the host; replaces
 * arma::auto_covariance (src/arma.cc:81-100), which the wave-group ACF
 * generator calls (src/generator/acf_generator.cc:147).  in and out may
 * alias. */
int arma_auto_covariance(const double* in, const int shape[3], double* out);
/* The same on the device for a surface in device memory (FP32 or FP64 per
 * `precision`; ARMA_FP32C reads FP32), the result in FP64 device memory: the
 * ACF of a realisation, as the reference checks generated surfaces.  Every
 * side <= 1024 (ARMA_ENOTSUP beyond); asynchronous on the context's stream. */
int arma_auto_covariance_device(arma_ctx* ctx, const void* d_in, const int shape[3],
                                int precision, double* d_out);
/* Analytic ACF on the non-negative lag grid (src/acf.hh:18-62). */
int arma_acf_eval(int kind, double amplitude, double velocity,
                  const double alpha[3], const double beta[2],
                  const double delta[3], const int shape[3], double* acf);
/* Gauss-elimination Yule-Walker fit on a tabulated ACF with the reference's
 * per-axis |lag| block-Toeplitz matrix (determine_coefficients_gauss,
 * src/generator/ar_model.cc:97-135; white_noise_variance :55-61). FP64. */
int arma_ar_fit(const double* acf, const int acf_shape[3], const int order[3],
                int method, double* phi, double* var_wn);
/* Same fit for an analytic ACF with the signed-lag matrix
 * R[p,q] = gamma(p - q) (an extension: equal to the reference's matrix for
 * standing waves; SPD for propagating waves, where the reference's |lag|
 * matrix is indefinite).  LL^T Cholesky, FP64. */
int arma_ar_fit_analytic(int kind, double amplitude, double velocity,
                         const double alpha[3], const double beta[2],
                         const double delta[3], const int order[3],
                         double* phi, double* var_wn);

/* ------------------------------------------------------ A7: white noise */
/* n normals N(0, stddev^2) in C order from one stream, as
 * prng::generate_white_noise + std::normal_distribution (Marsaglia polar over
 * generate_canonical) produce them (src/white_noise.hh:23-58,
 * src/generator/basic_arma_model.cc:36-48).  precision selects double or
 * float output (float = the double value rounded). */
int arma_white_noise(arma_ctx* ctx, const arma_mt_params* p, uint32_t seed,
                     double stddev, size_t n, int precision, void* d_out);

/* ------------------------------------------------------ A8: AR filter */
/* In-place causal AR filter over zeta holding the white noise
 * (ar_generate_surface, src/generator/ar_model_surf.cc:5-36; backend seam
 * AR_model::generate_surface, src/generator/ar_model.hh:102-103).
 * ARMA_FP64 follows the reference's summation order exactly;
 * ARMA_FP32C runs the compensated FP32 tile wavefront, for orders with
 * px <= 17, py <= 13 and pt * px <= 221 (others: ARMA_ENOTSUP).  Either
 * form takes orders of at most 16 per axis. */
int arma_ar_filter(arma_ctx* ctx, const double* phi, const int order[3],
                   const int shape[3], int precision, void* d_zeta);

/* Allocation-free variant of arma_ar_filter(..., ARMA_FP32C, ...) for one
 * surface: no counterpart in the reference.  For callers that cannot allocate
 * device memory on their calling path (code inside another framework's memory
 * pool, serving loops that forbid allocation, plugins whose host process owns
 * the device allocator).  It needs no context: work goes to `stream` (0 = the
 * legacy default stream) on the current device, and all scratch lives in one
 * 64 KiB __device__ array that every GPU loading the library holds until exit.
 * Limits: <= 2048 coefficients and <= 8192 tiles of 16x32 points per slice;
 * larger requests fail with ARMA_EINVAL; orders outside the FP32 kernel's
 * (see arma_ar_filter) with ARMA_ENOTSUP.  Its result is bit-identical to
 * arma_ar_filter(..., ARMA_FP32C, ...) on the same input (same coefficient
 * tables, same kernel).  The first call on a device looks up the array's
 * address (once per device, thread-safe).  Every call stages its tables from
 * host memory, reads the device error word back and synchronises `stream`,
 * so it cannot be used under stream capture: a capturing stream is refused
 * with ARMA_EINVAL.  Calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int arma_ar_filter_fp32c_noalloc(void* stream, const double* phi, const int order[3],
                                 const int shape[3], float* d_zeta);

/* One x-strip of a surface split by rows across devices, for a surface too
 * large for one device (the reference ships each partition of a surface with
 * its halo to a remote kernel, src/generator/ar_model_bscheduler.cc:285-353).
 * d_zeta holds shape = (nt, nx, ny): rows [0, given_rows) of every slice and
 * slices [0, t0) are given -- finished values (the last rows of the strip
 * above, zeros above the surface's first row; the previous time chunk) that
 * are read and never written -- and every other point holds its white noise
 * on entry and its surface value on return.  given_rows is 0 or a multiple
 * of the filter's 16 tile rows below nx; FP32C orders only (see
 * arma_ar_filter).  When the strip's first computed row sits at a multiple of
 * 16 rows of the whole surface, its rows are bit-identical to
 * arma_ar_filter(..., ARMA_FP32C, ...) of the whole surface. */
int arma_ar_filter_strip(arma_ctx* ctx, const double* phi, const int order[3],
                         const int shape[3], int t0, int given_rows, float* d_zeta);

/* ------------------------------------------ A10: variance renormalisation */
/* zeta *= sqrt(acf0 / var) with var the unbiased variance of the
 * numElements() contiguous values starting at zeta(nt/2, nx/2, ny/2)
 * (src/generator/basic_arma_model.cc:102-106). */
int arma_variance_renorm(arma_ctx* ctx, void* d_zeta, const int shape[3],
                         int precision, double acf0, double* scale_out);

/* ------------------------------------------------------------ A11: NIT */
/* In place over n values (NIT_transform::transform_realisation,
 * src/nonlinear/nit_transform.cc:127-168).  params: Gram-Charlier
 * {skewness, kurtosis(non-excess)}; skew normal {mean, stdev, alpha}.
 * ARMA_NIT_BISECTION reproduces the per-point bisection on `interval` with
 * absolute error eps and max_iter iterations; ARMA_NIT_LUT maps through an
 * inverse-CDF table of lut_nodes nodes over [-lut_range, lut_range]*stdev
 * built in FP64. */
int arma_nit_apply(arma_ctx* ctx, int dist, const double params[3],
                   double stdev, int method, const double interval[2],
                   double eps, int max_iter, int lut_nodes, double lut_range,
                   size_t n, int precision, void* d_zeta);

/* ------------------------------------------- V1-V5: linear velocity solver */
/* Velocity_potential_solver::operator() with the Linear_solver hooks
 * (src/velocity/basic_solver.cc:38-77, src/velocity/linear_solver.cc:20-184).
 * t_idx: integer slice indices (the reference truncates domain t values);
 * z: depth levels; depth may be +INFINITY.  d_phi_out: (ntd, nz, nx, ny). */
int arma_velocity_linear(arma_ctx* ctx, const void* d_zeta, const int shape[3],
                         int precision, const double delta[3], double depth,
                         const double* z, int nz, const int* t_idx, int ntd,
                         void* d_phi_out);
/* High_amplitude_solver (src/velocity/high_amplitude_solver.cc:7-23): the
 * linear solver's pipeline on the complex input d zeta/dt / (i ((zx + zy)/s -
 * zx - zy) - 1/s), s = sqrt(1 + zx^2 + zy^2), slopes zx, zy from delta[1],
 * delta[2].  Same arguments as arma_velocity_linear. */
int arma_velocity_high_amplitude(arma_ctx* ctx, const void* d_zeta, const int shape[3],
                                 int precision, const double delta[3], double depth,
                                 const double* z, int nz, const int* t_idx, int ntd,
                                 void* d_phi_out);

/* Many surfaces of one slice shape nx x ny in one set of launches (no
 * counterpart in the reference): job k reads nt slices at d_zeta and writes
 * its slices t_idx[0..ntd) to d_out as (ntd, nz, nx, ny); dt is its time step
 * (<= 0: 1). */
typedef struct {
	const void* d_zeta;
	void* d_out;
	int nt;
	const int* t_idx;
	int ntd;
	double dt;
} arma_velocity_job;
int arma_velocity_linear_batch(arma_ctx* ctx, const arma_velocity_job* jobs, int n, int nx,
                               int ny, int precision, double depth, const double* z, int nz);

/* ------------------------------------------------ batched generation */
/* One surface of a batch.  phi/var_wn come from a fit; the noise stream is
 * (mt, seed); zeta is a device buffer of shape[0]*shape[1]*shape[2] elements
 * of the batch precision.  acf0 > 0 enables the variance renormalisation. */
typedef struct {
	int shape[3];
	int order[3];
	const double* phi; /* host, pt*px*py */
	double var_wn;
	double acf0;
	arma_mt_params mt;
	uint32_t seed;
	void* d_zeta;
	double scale; /* out: renormalisation factor */
} arma_surface;

/* White noise + AR filter (+ renormalisation) for n independent surfaces.
 * ARMA_FP32C runs all surfaces in one persistent launch; ARMA_FP64 runs the
 * plain filter surface by surface. */
int arma_batch_generate(arma_ctx* ctx, arma_surface* surfaces, int n,
                        int precision);
/* Same, writing each surface into a HOST buffer (d_zeta is then a host
 * pointer of doubles); host<->device copies are part of the call. */
int arma_batch_generate_host(arma_ctx* ctx, arma_surface* surfaces, int n,
                             int precision);

/* Times candidate settings on this batch (arma_batch_generate, or
 * arma_batch_generate_host with host = 1; the surfaces' buffers are written)
 * by coordinate descent over the MT segment length, the filter's CTAs per SM
 * and, for host output, the group split; sets the fastest on the context and
 * returns it with its time per call.  The choice is cached per batch shape
 * class (precision, host, surface count and the histogram of slice sizes,
 * lengths and orders) for the life of the process: a later call on the same
 * class sets the cached setting without timing. */
int arma_autotune(arma_ctx* ctx, arma_surface* surfaces, int n, int precision, int host,
                  arma_tuning* best, double* best_ms);

/* The NIT of one batch surface: the inverse-CDF table of arma_nit_apply's
 * ARMA_NIT_LUT method (lut_nodes nodes over [-lut_range, lut_range] * stdev,
 * built in FP64). */
typedef struct {
	int dist;          /* ARMA_NIT_GRAM_CHARLIER or ARMA_NIT_SKEW_NORMAL; < 0: none */
	double params[3];  /* as arma_nit_apply */
	double stdev;      /* of the Gaussian input (sqrt(acf0) in the reference) */
	int lut_nodes;
	double lut_range;
} arma_nit_table;
/* arma_batch_generate followed by the NIT of each surface whose nit[k].dist
 * is >= 0, as Basic_ARMA_model::generate runs them (the variance
 * renormalisation, then NIT_transform::transform_realisation;
 * src/generator/basic_arma_model.cc:102-110, src/nonlinear/nit_transform.cc:
 * 127-168): the table is applied in the renormalisation's scale pass, one read
 * and one write per value, and the result equals arma_batch_generate followed
 * by arma_nit_apply(ARMA_NIT_LUT) bit for bit.  A surface with NIT needs
 * acf0 > 0 (the reference renormalises before the transform).  Tables are
 * built once per distinct specification and kept by the context. */
int arma_batch_generate_nit(arma_ctx* ctx, arma_surface* surfaces, int n,
                            int precision, const arma_nit_table* nit);

/* ------------------------------------------------ A3': Choi solver */
/* Yule_walker_solver::solve (src/yule_walker.cc:426-539) as called by
 * AR_model::determine_coefficients_choi (src/generator/ar_model.cc:136-152):
 * the order-recursive solver on a cubic acf of n^3 values (lags accessed by
 * absolute value), up to max_order (clamped to n-1); with determine_order it
 * stops when the white-noise variance changes by less than var_epsilon (the
 * reference's AR model uses 1e-6); with chop it drops trailing planes whose
 * values are all below 1e-10.  phi_out must hold max_order^3 doubles;
 * order_out receives the model's shape; var_wn = acf(0,0,0) - sum(phi * acf
 * over phi's box), as the reference recomputes it. */
int arma_ar_fit_choi(const double* acf, int n, int max_order, int determine_order,
                     double var_epsilon, int chop, double* phi_out, int order_out[3],
                     double* var_wn);

/* ------------------------------------------------ A5: stationarity */
/* validate_process (src/arma.cc:14-70): the roots of the flattened
 * polynomial 1 - sum_k phi_k x^k, k = 1 .. P-1 (P = order product), by the
 * balanced companion-matrix QR method of gsl_poly_complex_solve.  ARMA_OK when
 * every root lies outside the unit circle; ARMA_EINVAL otherwise ("AR/MA
 * process is not stationary/invertible..."), with *bad_roots set; ARMA_ENUMERIC
 * when the leading coefficient is zero or the iteration fails. */
int arma_validate_process(const double* phi, const int order[3], int* bad_roots);
/* The root finder itself: roots of c[0] + c[1] x + ... + c[n-1] x^(n-1) into
 * re/im (n-1 each), as gsl_poly_complex_solve. */
int arma_poly_roots(const double* c, int n, double* re, double* im);

/* ------------------------------------------------ M: moving-average model */
/* MA coefficients by fixed-point iteration: replaces
 * MA_coefficient_solver::solve_fixed_point_iteration
 * (src/generator/ma_coefficient_solver.cc:36-139) with its defaults
 * (max_iterations 1000, max_residual 1e-5, min white-noise variance 1e-6,
 * variance tolerance 1e-5; src/generator/ma_coefficient_solver.hh:27-40).
 * acf has acf_shape (t,x,y) values; order <= acf_shape per axis.  theta_out
 * receives order[0]*order[1]*order[2] doubles with theta(0,0,0) = -1;
 * var_wn = acf(0,0,0) / sum theta^2 (src/arma.cc:73-79); iterations may be
 * NULL.  ARMA_EINVAL "bad order"; ARMA_ENUMERIC "bad MA model coefficients"
 * (non-finite) or "bad white noise variance" (at or below 1e-6). */
int arma_ma_fit(const double* acf, const int acf_shape[3], const int order[3],
                double* theta_out, double* var_wn, int* iterations);
/* The MA filter on device buffers of `precision`: zeta = eps - sum over
 * m != 0 of theta(m) eps(n - m), zero history; replaces
 * MA_model::generate_surface (src/generator/ma_model.cc:42-61, FFT
 * convolution with K = -theta, K(0,0,0) = 1).  theta is host, order-box
 * sized (theta(0,0,0) is ignored); d_eps and d_zeta must not overlap. */
int arma_ma_filter(arma_ctx* ctx, const double* theta, const int order[3],
                   const int shape[3], int precision, const void* d_eps, void* d_zeta);
/* White noise + MA filter (+ renormalisation) for n surfaces, as
 * arma_batch_generate with surfaces[k].phi holding theta: MA_model::do_generate
 * (src/generator/ma_model.cc:30-40) followed by the variance renormalisation
 * of Basic_ARMA_model::generate (src/generator/basic_arma_model.cc:98-103). */
int arma_ma_generate(arma_ctx* ctx, arma_surface* surfaces, int n, int precision);

/* ------------------------------------------------ programme layer */
/* The reference's ARMA_driver (src/arma_driver.hh:43-150): parses a `.arma`
 * configuration (`model = AR {...}`, `velocity_potential_solver = linear |
 * high_amplitude {...}`; the other registered names return ARMA_ENOTSUP; `acf = {...}`
 * without `grid` is the reference's wave-group ACF_generator, with `grid` the
 * analytic standing / propagating ACF), runs
 * generate_wavy_surface / compute_velocity_potentials on the device, and
 * writes zeta / zeta.csv / zeta.bin / phi / phi.csv like write_all
 * (src/arma_driver.cc:29-178).  Extensions: `seed`, `mt_file`,
 * `precision = fp64|fp32c`, `depth = inf`, `z_levels = [..]`. */
typedef struct arma_driver arma_driver;
int arma_driver_open(const char* config, int is_path, arma_driver** out);
int arma_driver_close(arma_driver* drv);
/* Failure-path self-test: runs the FP32 filter's bounded neighbour wait on a
 * tile flag that nothing publishes; the wait gives up after its poll limit
 * (about a second), the call returns ARMA_ETIMEDOUT, and the context stays
 * usable (its error word is cleared). */
int arma_selftest_wait(arma_ctx* ctx);
/* Directory of the files written while generating (default: the working
 * directory, as the reference): with the `binary` flag an AR model's zeta.bin
 * is streamed there in t-slabs during arma_driver_generate, holding the
 * surface before the variance renormalisation and the NIT, as the
 * reference's writer thread writes it (src/generator/ar_model_parallel.cc:
 * 112-145, joined at :196-198 before src/generator/basic_arma_model.cc:106);
 * arma_driver_write_all then does not write it again. */
int arma_driver_set_output_dir(arma_driver* drv, const char* dir);
int arma_driver_generate(arma_ctx* ctx, arma_driver* drv);
int arma_driver_compute_velocity(arma_ctx* ctx, arma_driver* drv);
int arma_driver_write_all(arma_driver* drv, const char* dir);
/* shape/delta of zeta, AR order, white-noise variance, velocity shape
 * (nt_dom, nz, nx, ny) and the output flags (bit k = flag k of none,
 * summary, qq, waves, acf, csv, blitz, binary, surface as in
 * src/output_flags.cc:13-23); any pointer may be null. */
int arma_driver_info(arma_driver* drv, int shape[3], double delta[3], int order[3],
                     double* var_wn, int vshape[4], unsigned* output_flags);
/* Copies zeta (what = 0), phi coefficients (1) or velocity potentials (2). */
int arma_driver_copy(arma_driver* drv, int what, double* out);
/* The model's ACF table (available after open): its shape and grid step, and
 * the values into out when out is not NULL. */
int arma_driver_acf(arma_driver* drv, int shape[3], double delta[3], double* out);

/* ------------------------------------------------ serving */
/* No counterpart in the reference.  A server owns device-resident surface
 * streams: each stream is an unbounded surface of fixed nx x ny with one AR
 * model (FP32 compensated filter) and one dcmt stream, generated in chunks of
 * chunk_slices time slices.  A stream's chunks concatenated equal one surface
 * generated in a single call with the same seed; with acf0 > 0 every chunk is
 * scaled by the renormalisation factor of the first chunk.  Requests for the
 * next chunk of any stream are batched continuously by a host thread (up to
 * max_inflight device batches overlap) and admitted by the HBM footprint of
 * the stream state (two slice buffers of pt-1+chunk_slices slices, the MT
 * window, velocity and output staging). */
typedef struct arma_server arma_server;
typedef struct {
	int chunk_slices;           /* T, even (default 64) */
	int max_inflight;           /* device batches in flight, 1..8 (default 3) */
	int max_batch;              /* requests per batch (default 64) */
	long long max_batch_points; /* surface points per batch (default 2^26) */
	size_t hbm_budget;          /* bytes of stream state (0: half the free memory) */
	int velocity;               /* 1: velocity potentials of every chunk slice */
	double depth;               /* velocity solver depth (INFINITY allowed) */
	int nz;                     /* number of z levels, 1..8 */
	double z_levels[8];
	double noise_margin;        /* multiplier of the polar-attempt estimate (1) */
	int profile;                /* 1: time kernel classes with CUDA events */
} arma_server_config;

typedef struct {
	int nx, ny;
	int order[3];          /* pt, px, py */
	const double* phi;     /* FP64 coefficients, copied at open */
	double var_wn;
	double acf0;           /* > 0: renormalise by the first chunk */
	arma_mt_params mt;
	uint32_t seed;
	double delta[3];       /* grid steps (t, x, y) for the velocity solver */
} arma_stream_spec;

typedef struct {
	uint64_t request, stream, chunk;
	int status;            /* ARMA_OK or an error code */
	int batch_size;        /* requests in the device batch that ran it */
	double latency_ms;     /* submit -> outputs in place */
	double queue_ms;       /* submit -> launch */
	double device_ms;      /* the batch's time on the GPU */
} arma_completion;

typedef struct {
	uint64_t submitted, completed, batches, redone, launches;
	uint64_t points;       /* surface points delivered */
	size_t resident_bytes, budget_bytes;
	int streams, resident_streams, inflight, pending;
	double launch_ms_total, launch_ms_max;  /* host time spent enqueueing batches */
} arma_server_stats;

int arma_server_config_default(arma_server_config* cfg);
int arma_server_create(int device, const arma_server_config* cfg, arma_server** out);
/* Finishes every queued request, then frees everything. */
int arma_server_destroy(arma_server* srv);
int arma_stream_open(arma_server* srv, const arma_stream_spec* spec, uint64_t* stream_id);
/* The stream's memory is released once its queued requests are done. */
int arma_stream_close(arma_server* srv, uint64_t stream_id);
/* Queues the stream's next chunk.  zeta_out: chunk_slices*nx*ny floats;
 * velocity_out: chunk_slices*nz*nx*ny floats (t, z, x, y) or NULL.  Both must
 * be device memory or page-locked host memory and stay valid until the
 * request completes. */
int arma_stream_submit(arma_server* srv, uint64_t stream_id, float* zeta_out,
                       float* velocity_out, uint64_t* request_id);
/* Up to max completions; waits up to timeout_ms (-1: forever) for the first. */
int arma_server_poll(arma_server* srv, arma_completion* out, int max, int timeout_ms, int* n);
int arma_server_stats_get(arma_server* srv, arma_server_stats* out);
/* With profile = 1: device milliseconds and scopes of one kernel class
 * ("mt", "noise", "ar32c", "renorm", "velocity", "copy") over idle slots. */
int arma_server_profile(arma_server* srv, const char* name, double* ms, uint64_t* launches);
/* The last failure the serving thread saw (empty if none). */
int arma_server_last_failure(arma_server* srv, char* buf, size_t len);

/* ------------------------------------------------ replica router */
/* No counterpart in the reference.  One server per listed device (a replica;
 * a device may be listed more than once) behind one handle, for serving on
 * several GPUs of a node: a stream opens on the replica with the least
 * stream state placed on it (nx * ny * (pt - 1 + 2 chunk_slices) points,
 * ties to fewer streams, then to the lower index) and stays there; its
 * requests go to that replica, and one poll returns the completions of all
 * replicas.  Stream and request ids are the replica's own ids with the
 * replica index in the top 8 bits, so ids of different replicas never
 * collide.  Replicas share nothing: no collective, no peer memory. */
typedef struct arma_router arma_router;
int arma_router_create(const int* devices, int n, const arma_server_config* cfg,
                       arma_router** out);
/* Destroys every replica (each finishes its queued requests first). */
int arma_router_destroy(arma_router* r);
int arma_router_replicas(arma_router* r, int* n);
int arma_router_stream_open(arma_router* r, const arma_stream_spec* spec, uint64_t* stream_id);
int arma_router_stream_close(arma_router* r, uint64_t stream_id);
/* As arma_stream_submit; the outputs must be memory of the stream's replica's
 * device (or page-locked host memory). */
int arma_router_stream_submit(arma_router* r, uint64_t stream_id, float* zeta_out,
                              float* velocity_out, uint64_t* request_id);
/* Up to max completions of any replica; waits up to timeout_ms (-1: forever)
 * for the first. */
int arma_router_poll(arma_router* r, arma_completion* out, int max, int timeout_ms, int* n);
/* The replica index and device a stream was placed on. */
int arma_router_placement(arma_router* r, uint64_t stream_id, int* replica, int* device);
int arma_router_stats_get(arma_router* r, int replica, arma_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* ARMA_B200_H */
