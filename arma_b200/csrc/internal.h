// Internal declarations shared by the C-ABI layer and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <exception>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/arma_b200.h"

namespace armab {

// ------------------------------------------------------------- errors
void set_error(const std::string& msg);
const std::string& last_error();

struct Error {
	int code;
	std::string msg;
};

#define ARMA_CUDA_TRY(expr)                                                         \
	do {                                                                            \
		cudaError_t e_ = (expr);                                                    \
		if (e_ != cudaSuccess)                                                      \
			throw ::armab::Error{ARMA_ECUDA, std::string(#expr) + ": " +            \
			                                     cudaGetErrorString(e_)};          \
	} while (0)

#define ARMA_REQUIRE(cond, code, msg)                                               \
	do {                                                                            \
		if (!(cond)) throw ::armab::Error{(code), (msg)};                           \
	} while (0)

// Device-side error word values (bounded waits and checks write these).
enum DeviceError : int {
	DEV_OK = 0,
	DEV_TIMEOUT = 1,
	DEV_BOUNDS = 2,
};

// ------------------------------------------------------------- context
struct Ctx {
	int device = 0;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	int* d_err = nullptr;            // device error word
	cudaStream_t copy_stream = nullptr;  // device->host copies overlapped with compute (lazy)
	cudaStream_t side_stream = nullptr;  // second compute stream of the host-output pipeline (lazy)
	double noise_margin = 1.0;           // polar-attempt estimate multiplier of the batched calls
	arma_tuning tuning{20, 0, 16, 0.06};  // result-invariant speed settings (arma_ctx_set_tuning)
	uint64_t launches = 0;           // kernel launches issued
	uint64_t h2d_bytes = 0;          // bytes copied host -> device through copy_async
	uint64_t d2h_bytes = 0;          // bytes copied device -> host through copy_async
	int num_sms = 148;
	// cached CUDA graphs for the FP64 plane sweep, keyed by a string
	std::map<std::string, cudaGraphExec_t> graphs;
	// NIT inverse-CDF tables by specification (double table, then float table)
	std::map<std::vector<double>, double*> nit_tables;
	// optional per-kernel-class timing with CUDA events on `stream`
	bool profiling = false;
	struct Pending {
		std::string name;
		cudaEvent_t start, stop;
	};
	std::vector<Pending> pending;
	std::map<std::string, double> prof_ms;
	std::map<std::string, long long> prof_count;
};

// The NIT table map shared by the standalone NIT kernel and the fused
// renormalisation.  With u = (z - x0) / dx the table holds, for each interval
// u in [j, j + 1) (j = 0 .. nodes-2), the power-basis coefficients in
// t = u - j of the cubic Lagrange interpolant through nodes i-1 .. i+2
// (i = clamp(j, 1, nodes-3)), and at j = nodes-1 and j = nodes the linear
// extrapolations beyond the first and the last node (value and node step).
// One vector load and three FMAs per value.
template <class T> struct NitCoef;
template <> struct NitCoef<float> { using type = float4; };
template <> struct NitCoef<double> { using type = double4; };

template <class T>
__device__ __forceinline__ T nit_lut_map(T z, const typename NitCoef<T>::type* __restrict__ coef,
                                         int nodes, T x0, T inv_dx) {
	const T u = (z - x0) * inv_dx;
	int j;
	T t;
	if (u <= T(0)) {
		j = nodes - 1;
		t = u;
	} else if (u >= T(nodes - 1)) {
		j = nodes;
		t = u - T(nodes - 1);
	} else {
		j = min(int(u), nodes - 2);
		t = u - T(j);
	}
	const typename NitCoef<T>::type k = coef[j];
	return fma(fma(fma(k.w, t, k.z), t, k.y), t, k.x);
}

// cudaMemcpyAsync that counts the bytes a context moves between host and
// device (arma_ctx_transfer_bytes).
inline cudaError_t copy_async(Ctx* c, void* dst, const void* src, size_t bytes,
                              cudaMemcpyKind kind, cudaStream_t stream) {
	if (kind == cudaMemcpyHostToDevice) c->h2d_bytes += bytes;
	if (kind == cudaMemcpyDeviceToHost) c->d2h_bytes += bytes;
	return cudaMemcpyAsync(dst, src, bytes, kind, stream);
}

// Records CUDA events around a launch when profiling is on.
class ProfScope {
public:
	ProfScope(Ctx* c, const char* name);
	~ProfScope();
private:
	Ctx* c_;
	int idx_ = -1;
};
void resolve_profile(Ctx* c);

// Device scratch: a bump arena of chunks owned by the context.  scratch_take
// returns 256-byte aligned memory valid until the next scratch_begin (the start
// of the next API call); a call that outgrows the current chunk gets a new
// chunk, and the next scratch_begin merges the chunks into one of the
// high-water size (synchronising the stream first).
void scratch_begin(Ctx* c, size_t total_bytes);
void* scratch_take(Ctx* c, size_t bytes);
// Work enqueued in order on the context's stream may reuse scratch: take a
// mark, enqueue, release back to the mark.
struct ScratchMark {
	size_t chunks, used, taken;
};
ScratchMark scratch_mark(Ctx* c);
// Grows the arena to at least `bytes` in one chunk now, so that later calls
// of up to that size never allocate.
void scratch_reserve(Ctx* c, size_t bytes);
void scratch_release(Ctx* c, const ScratchMark& m);
// The library's stream-ordered device memory pool (one per device; freed
// blocks are kept for reuse).  Allocations are ordered on c->stream.
void* pool_alloc(Ctx* c, size_t bytes);
void pool_free(Ctx* c, void* p);

void check_device_error(Ctx* c);

// ------------------------------------------------------------- launchers
// MT: tempered words [offset, offset+n) of stream (p, seed) into d_out.  A job
// with `state` set starts from that raw window of nn words instead of the
// seeded state (offset must then be 0).
struct MtJob {
	arma_mt_params p;
	uint32_t seed;
	unsigned long long offset, count;
	uint32_t* out;
	const uint32_t* state = nullptr;
	// the windows at every segment start (launch_mt_prepare with the same
	// segment length), or null: jump ahead here
	const uint32_t* seg_states = nullptr;
};
void launch_mt_generate(Ctx* c, const arma_mt_params& p, uint32_t seed,
                        uint64_t offset, uint64_t n, uint32_t* d_out);
// Every job's stream in a few launches: streams longer than one segment of
// 2^log2_seg words are split by jump-ahead into one CTA per segment.
constexpr int kMtLog2Seg = 20;
void launch_mt_generate_batch(Ctx* c, const std::vector<MtJob>& jobs,
                              int log2_seg = kMtLog2Seg);
// Only the jump-ahead windows of the jobs longer than one segment, into
// jobs[q].seg_states (scratch), for later launch_mt_generate_batch calls on
// subsets of the jobs with the same segment length.
void launch_mt_prepare(Ctx* c, std::vector<MtJob>& jobs, int log2_seg = kMtLog2Seg);
// After a chunk consumed 4 * *attempts words of `words` (n_words long): the
// raw window in front of the next word (untempered copies of the nn words
// before it), and *position += 4 * *attempts.  All on the device; an attempt
// count outside [nn/4, n_words/4] (0: the noise ran short) changes nothing.
struct MtWindowSpec {
	arma_mt_params p;
	const uint32_t* words;
	unsigned long long n_words;
	const unsigned long long* attempts;
	uint32_t* window;
	unsigned long long* position;
};
void launch_mt_window_update(Ctx* c, const std::vector<MtWindowSpec>& specs);

// White noise: n normals from the word stream d_words (n_words words).
// enqueue_white_noise writes the number of accepted pairs to *d_pairs and does
// not synchronise; launch_white_noise synchronises and returns false when the
// words did not contain enough accepted pairs.
void enqueue_white_noise(Ctx* c, const uint32_t* d_words, uint64_t n_words,
                         double stddev, uint64_t n, int precision, void* d_out,
                         long long* d_pairs);
bool launch_white_noise(Ctx* c, const uint32_t* d_words, uint64_t n_words,
                        double stddev, uint64_t n, int precision, void* d_out);
// All surfaces of a batch in three launches; d_pairs[k] receives surface k's
// number of accepted pairs (no synchronisation).
// With `attempts` set (n even), the index + 1 of the polar attempt that gave
// the last pair is written there: the words the noise consumed are 4 times it.
struct NoiseSpec {
	const uint32_t* words;
	uint64_t n_words;
	uint64_t n;
	double stddev;
	void* out;
	unsigned long long* attempts = nullptr;
};
void enqueue_white_noise_batch(Ctx* c, const std::vector<NoiseSpec>& specs, int precision,
                               long long* d_pairs);

// FP64 exact-order AR filter.
void launch_ar64(Ctx* c, const double* d_phi, const int order[3],
                 const int shape[3], double* d_zeta);

// FP32 compensated AR filter for a batch of surfaces (ar32c.cu).
struct Ar32Surface {
	int nt, nx, ny;
	int pt, px, py;
	float* zeta;           // device, in place (noise in, surface out)
	const float* phi;      // device, pt*px*py, hi part of the FP64 coefficients
	const float* phi_lo;   // device, pt*px*py, phi - hi
	const float* h;        // device, intra-slice impulse response (TX*TY)
	int tiles_x, tiles_y;  // spatial tile grid
	int t0 = 0;            // slices [0, t0) hold a finished history (streams)
	int given_tx = 0;      // tile rows [0, given_tx) hold given values (x-strips)
};
void launch_ar32c(Ctx* c, const std::vector<Ar32Surface>& surfaces, int tx,
                  int ty, int tt);
// One bounded neighbour wait of the FP32 filter on a flag nothing sets
// (arma_selftest_wait); leaves DEV_TIMEOUT in the context's error word.
void launch_wait_selftest(Ctx* c);
int ar32c_tile_x();
int ar32c_tile_y();
int ar32c_max_tap_rows();  // largest pt * px of the FP32 tile kernel

// Variance renormalisation: computes scale on device (d_scale) and applies it.
void launch_renorm(Ctx* c, void* d_zeta, const int shape[3], int precision,
                   double acf0, double* d_scale);
struct RenormSpec {
	void* z;
	int shape[3];
	double acf0;
	double* d_scale;
	// optional NIT inverse-CDF table applied right after the scale (same
	// element type as the surface; nullptr: none)
	const void* lut = nullptr;
	int lut_nodes = 0;
	double lut_x0 = 0.0, lut_inv_dx = 0.0;
};
// apply = false only computes the scales.
void launch_renorm_batch(Ctx* c, const std::vector<RenormSpec>& specs, int precision,
                         bool apply = true);

// NIT.
void launch_nit_bisection(Ctx* c, int dist, const double params[3], double stdev,
                          double a, double b, double eps, int max_iter,
                          uint64_t n, int precision, void* d_zeta);
// d_coef: the table of nit_lut_coefficients in the call's precision
// (4 (nodes + 1) values).
void launch_nit_lut(Ctx* c, const void* d_coef, int nodes, double x0,
                    double dx, uint64_t n, int precision, void* d_zeta);

// Velocity.
// mode 0: the linear solver; mode 1: the high-amplitude solver (slopes from
// delta[1], delta[2]).
void launch_velocity_linear(Ctx* c, const void* d_zeta, const int shape[3],
                            int precision, const double delta[3], double depth,
                            const double* z, int nz, const int* t_idx, int ntd,
                            void* d_out, int mode = 0);
// Many surfaces of one slice shape nx x ny in one set of launches: surface k
// has nt slices at zeta, its slices t_idx[0..ntd) go to out as (ntd, nz, nx,
// ny); dt is its time step.
struct VelocitySurface {
	const void* zeta;
	void* out;
	int nt;
	const int* t_idx;
	int ntd;
	double dt;
	int mode = 0;               // 0 linear, 1 high amplitude
	double dx = 1.0, dy = 1.0;  // steps for the slopes of mode 1
};
void launch_velocity_linear_batch(Ctx* c, const VelocitySurface* v, int n, int nx, int ny,
                                  int precision, double depth, const double* z, int nz);
// Slice shapes the solver's FFTs take: sides in [4, 1024], prime factors <= 64.
bool velocity_supported(int nx, int ny);

// Host math shared by the ABI (fit.cc).
int fit_gauss_table(const double* acf, const int acf_shape[3], const int order[3],
                    int method, double* phi, double* var_wn);
int fit_analytic(int kind, double amplitude, double velocity, const double alpha[3],
                 const double beta[2], const double delta[3], const int order[3],
                 double* phi, double* var_wn);
void acf_eval(int kind, double amplitude, double velocity, const double alpha[3],
              const double beta[2], const double delta[3], const int shape[3],
              double* out);
// Intra-slice impulse response of 1 / (1 - sum phi(0,i,j) z1^-i z2^-j) on a
// tx x ty quarter plane, FP64.
void intra_slice_response(const double* phi, const int order[3], int tx, int ty,
                          double* h);
// White noise + AR filter (+ renormalisation) into device buffers (capi.cu).
void batch_generate_device(Ctx* c, arma_surface* s, int n, int precision);
// The MA form: s[k].phi holds theta (noise, MA filter, renormalisation).
void ma_generate_device(Ctx* c, arma_surface* s, int n, int precision);

// The `.arma` programme layer (driver.cc).
struct Driver;
Driver* driver_open(const std::string& text);
void driver_close(Driver* d);
void driver_generate(Ctx* c, Driver* d);
void driver_velocity(Ctx* c, Driver* d);
void driver_write(Driver* d, const std::string& dir);
void driver_set_output_dir(Driver* d, const std::string& dir);
void driver_info(const Driver* d, int shape[3], double delta[3], int order[3], double* var_wn,
                 int vshape[4], unsigned* oflags);
const double* driver_zeta(const Driver* d);
void driver_acf(const Driver* d, int shape[3], double delta[3], const double** data);
const double* driver_phi(const Driver* d);
const double* driver_velocity_data(const Driver* d);

// Inverse-CDF table for the NIT LUT path.
void nit_build_lut(int dist, const double params[3], double stdev, int nodes,
                   double range, double* x0, double* dx, std::vector<double>& y);
// The device form of a table of y.size() >= 4 nodes: 4 (nodes + 1) values,
// the per-interval cubic coefficients and the two end extrapolations that
// nit_lut_map reads.
std::vector<double> nit_lut_coefficients(const std::vector<double>& y);

// The empirical ACF of a plain-wave group (acf_gen.cc): func 0 sin, 1 cos,
// 2 stokes, 3 standing wave; wavenum = (kx, ky); shape = ACF shape (a zero
// component selects the doubling search).  Returns the ACF table and its shape
// and grid step.
struct EmpiricalAcf {
	int func = 1;
	double amplitude = 1.0, velocity = 1.0;
	double wavenum[2] = {0.8, 0.0};
	double alpha[3] = {0.06, 0.06, 0.06};
	double nwaves[3] = {1.5, 1.5, 1.5};
	int shape[3] = {16, 16, 16};
};
std::vector<double> empirical_acf(const EmpiricalAcf& p, int shape[3], double delta[3]);
std::vector<double> auto_covariance(const std::vector<double>& w, const int n[3]);
// The same on the device: d_in (FP32 or FP64, precision) -> d_out (FP64);
// sides <= 1024.
void launch_auto_covariance(Ctx* c, const void* d_in, const int shape[3], int precision,
                            double* d_out);

// Choi's order-recursive Yule-Walker solver (choi.cc) on a cubic n^3 ACF:
// 0 with phi (order[0] x order[1] x order[2]) and the solver's variance, 1 bad
// sizes, 2 singular block.
int fit_choi(const double* acf, int n, int max_order, bool determine_order, double var_eps,
             bool chop, double chop_eps, std::vector<double>* phi, int order[3], double* var_out);
// white_noise_variance (src/generator/ar_model.cc:55-61): acf(0,0,0) minus the
// sum of phi times the ACF over phi's box (acf is n0 x n1 x n2).
double ar_white_noise_variance(const double* acf, const int acf_shape[3], const double* phi,
                               const int order[3]);

// Roots of c[0] + c[1] x + ... + c[n-1] x^(n-1) (validate.cc): 0, 1 when the
// leading coefficient is zero or n < 2, 2 when the QR iteration does not
// converge.
int poly_roots(const double* c, int n, std::vector<std::complex<double>>& roots);
// validate_process on the flattened phi (P coefficients): 0 stationary, 3 with
// *bad_roots roots of modulus <= 1, or poly_roots' failure code.
int validate_ar_process(const double* phi, int P, int* bad_roots);

// MA coefficients by fixed-point iteration (ma_fit.cc), the solver's defaults
// (src/generator/ma_coefficient_solver.hh:27-40).
struct MaFitOptions {
	int max_iterations = 1000;
	double max_residual = 1e-5;
	double min_var_wn = 1e-6;
	double eps = 1e-5;
};
// 0 with theta (order box, theta(0,0,0) = -1) and var_wn; 1 order outside the
// ACF; 2 non-finite coefficients; 3 white-noise variance at or below the
// minimum (*var_out holds it).
int ma_fit_fixed_point(const double* acf, const int acf_shape[3], const int order[3],
                       const MaFitOptions& opt, std::vector<double>* theta_out, double* var_out,
                       int* iterations, double* residual_out);
// acf(0,0,0) / sum theta^2 (src/arma.cc:73-79).
double ma_white_noise_variance(const double* acf, const double* theta, const int order[3]);
// zeta = eps - sum_{m != 0} theta(m) eps(n - m) on the device (ma.cu); eps and
// zeta must not overlap.
void launch_ma_filter(Ctx* c, const double* theta, const int order[3], const int shape[3],
                      int precision, const void* d_eps, void* d_zeta);

// Polar attempts generated for n normals: the expected count plus 8 sigma,
// times `margin` (capi.cu).
uint64_t noise_attempts(size_t n, double margin);
void require_mt(const arma_mt_params* p);
// The FP32 tile kernel's coefficient block of one surface: phi hi, phi lo,
// H (ar32_coefficient_count floats).
size_t ar32_coefficient_count(const int order[3]);
void ar32_coefficients(const double* phi, const int order[3], float* out);

// dcmt parameter-set creation (dcmt.cpp).
namespace dcmt {
bool mersenne_exponent(int p);
bool is_primitive(const arma_mt_params& prm);
long equidistribution(const arma_mt_params& prm, int v);  // k(v), -1 if undetermined
int create(int p, int id, uint32_t seed, arma_mt_params* out);  // 0, or -1: no primitive set
}  // namespace dcmt

// Runs f, mapping library exceptions to status codes and the thread's last
// error message.
template <class F>
int guard(F&& f) {
	try {
		f();
		return ARMA_OK;
	} catch (const Error& e) {
		set_error(e.msg);
		return e.code;
	} catch (const std::bad_alloc&) {
		set_error("host allocation failed");
		return ARMA_ENOMEM;
	} catch (const std::exception& e) {
		set_error(e.what());
		return ARMA_EINVAL;
	}
}

}  // namespace armab

// The context behind the opaque arma_ctx handle.
struct arma_ctx {
	armab::Ctx c;
	std::vector<std::pair<char*, size_t>> chunks;  // scratch chunks
	size_t used = 0;                                // bytes used in the last chunk
	size_t high_water = 0;                          // total bytes taken in one call
	size_t taken = 0;
};
