// Internal declarations shared by the C-ABI layer and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
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
	uint64_t launches = 0;           // kernel launches issued
	int num_sms = 148;
	// cached CUDA graphs for the FP64 plane sweep, keyed by a string
	std::map<std::string, cudaGraphExec_t> graphs;
	// MT jump tables per parameter set: set-bit lists of t^(J 2^l) mod phi
	struct MtTable {
		bool ok = false;
		std::vector<int32_t*> bits;  // device arrays, one per level
		std::vector<int> nbits;
	};
	std::map<std::vector<uint32_t>, MtTable> mt_tables;
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

void check_device_error(Ctx* c);

// ------------------------------------------------------------- launchers
// MT: tempered words [offset, offset+n) of stream (p, seed) into d_out.
struct MtJob {
	arma_mt_params p;
	uint32_t seed;
	unsigned long long offset, count;
	uint32_t* out;
};
void launch_mt_generate(Ctx* c, const arma_mt_params& p, uint32_t seed,
                        uint64_t offset, uint64_t n, uint32_t* d_out);
// One launch generating every job's stream (one CTA per job).
void launch_mt_generate_batch(Ctx* c, const std::vector<MtJob>& jobs);

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
struct NoiseSpec {
	const uint32_t* words;
	uint64_t n_words;
	uint64_t n;
	double stddev;
	void* out;
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
	const float* h;        // device, intra-slice impulse response (TX*TY), hi
	const float* h_lo;     // device, lo part of h
	int tiles_x, tiles_y;  // spatial tile grid
};
void launch_ar32c(Ctx* c, const std::vector<Ar32Surface>& surfaces, int tx,
                  int ty, int tt);
int ar32c_tile_x();
int ar32c_tile_y();

// Variance renormalisation: computes scale on device (d_scale) and applies it.
void launch_renorm(Ctx* c, void* d_zeta, const int shape[3], int precision,
                   double acf0, double* d_scale);
struct RenormSpec {
	void* z;
	int shape[3];
	double acf0;
	double* d_scale;
};
void launch_renorm_batch(Ctx* c, const std::vector<RenormSpec>& specs, int precision);

// NIT.
void launch_nit_bisection(Ctx* c, int dist, const double params[3], double stdev,
                          double a, double b, double eps, int max_iter,
                          uint64_t n, int precision, void* d_zeta);
void launch_nit_lut(Ctx* c, const double* d_lut_y, int nodes, double x0,
                    double dx, uint64_t n, int precision, void* d_zeta);

// Velocity.
void launch_velocity_linear(Ctx* c, const void* d_zeta, const int shape[3],
                            int precision, const double delta[3], double depth,
                            const double* z, int nz, const int* t_idx, int ntd,
                            void* d_out);

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

// The `.arma` programme layer (driver.cc).
struct Driver;
Driver* driver_open(const std::string& text);
void driver_close(Driver* d);
void driver_generate(Ctx* c, Driver* d);
void driver_velocity(Ctx* c, Driver* d);
void driver_write(Driver* d, const std::string& dir);
void driver_info(const Driver* d, int shape[3], double delta[3], int order[3], double* var_wn,
                 int vshape[4], unsigned* oflags);
const double* driver_zeta(const Driver* d);
const double* driver_phi(const Driver* d);
const double* driver_velocity_data(const Driver* d);

// Inverse-CDF table for the NIT LUT path.
void nit_build_lut(int dist, const double params[3], double stdev, int nodes,
                   double range, double* x0, double* dx, std::vector<double>& y);

}  // namespace armab
