// Circular auto-covariance of a 3-D array on the device: the reference's
// arma::auto_covariance (src/arma.cc:81-100), Re IFFT(|FFT(w)|^2) / n / n,
// which its wave-group ACF generator (src/generator/acf_generator.cc:147) and
// its ACF checks of generated surfaces use.
//
// FP64 throughout.  The 3-D transform is one pass per axis; a CTA transforms
// one line: the line and the line's twiddles exp(+-2 pi i k / n) are staged in
// shared memory and each thread forms outputs q by direct summation (n^2
// complex multiply-adds per line, the twiddle index p q mod n kept as a running
// sum).  Lines of up to kMaxLine points: the reference's ACF generator works
// on 2 nwaves + 1 <= 129 points per axis, and a realisation's ACF check on its
// own sides (<= 1024).
#include <cmath>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr int kAcThreads = 256;
constexpr int kMaxLine = 1024;

// w[i] = (double) in[i] as a complex value
template <class T>
__global__ void to_complex_kernel(const T* __restrict__ in, double2* __restrict__ w,
                                  unsigned long long n) {
	for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
	     i += (unsigned long long)gridDim.x * blockDim.x)
		w[i] = make_double2(double(in[i]), 0.0);
}

// One line of n points along an axis whose points are `inner` apart: line b
// starts at (b / inner) n inner + b % inner.  In place: the line is read into
// shared memory before any output is written.
__global__ void __launch_bounds__(kAcThreads)
dft_axis_kernel(double2* __restrict__ d, int n, long long inner, double sign) {
	extern __shared__ double2 ac_smem[];
	double2* line = ac_smem;
	double2* tw = ac_smem + n;
	const long long b = blockIdx.x;
	double2* base = d + (b / inner) * (long long)n * inner + b % inner;
	for (int p = threadIdx.x; p < n; p += blockDim.x) {
		line[p] = base[p * inner];
		double s, c;
		sincospi(2.0 * p / n, &s, &c);
		tw[p] = make_double2(c, sign * s);
	}
	__syncthreads();
	for (int q = threadIdx.x; q < n; q += blockDim.x) {
		double re = 0.0, im = 0.0;
		int k = 0;  // p q mod n
		for (int p = 0; p < n; ++p) {
			const double2 x = line[p], w = tw[k];
			re = fma(x.x, w.x, fma(-x.y, w.y, re));
			im = fma(x.x, w.y, fma(x.y, w.x, im));
			k += q;
			if (k >= n) k -= n;
		}
		base[q * inner] = make_double2(re, im);
	}
}

__global__ void power_kernel(double2* __restrict__ w, unsigned long long n) {
	for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
	     i += (unsigned long long)gridDim.x * blockDim.x) {
		const double2 v = w[i];
		w[i] = make_double2(v.x * v.x + v.y * v.y, 0.0);
	}
}

__global__ void real_scaled_kernel(const double2* __restrict__ w, double* __restrict__ out,
                                   unsigned long long n, double nn) {
	for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
	     i += (unsigned long long)gridDim.x * blockDim.x)
		out[i] = w[i].x / nn / nn;
}

int flat_grid(Ctx* c, unsigned long long n) {
	const unsigned long long b = (n + kAcThreads - 1) / kAcThreads;
	const unsigned long long cap = 8ull * c->num_sms;
	return int(b < cap ? (b ? b : 1) : cap);
}

}  // namespace

void launch_auto_covariance(Ctx* c, const void* d_in, const int shape[3], int precision,
                            double* d_out) {
	ProfScope prof_(c, "autocov");
	for (int a = 0; a < 3; ++a)
		ARMA_REQUIRE(shape[a] >= 1 && shape[a] <= kMaxLine, ARMA_ENOTSUP,
		             "auto-covariance: sides must be in [1, 1024]");
	const unsigned long long n = (unsigned long long)shape[0] * shape[1] * shape[2];
	auto* w = static_cast<double2*>(scratch_take(c, sizeof(double2) * n));
	const int g = flat_grid(c, n);
	if (precision == ARMA_FP64)
		to_complex_kernel<double><<<g, kAcThreads, 0, c->stream>>>(static_cast<const double*>(d_in), w, n);
	else
		to_complex_kernel<float><<<g, kAcThreads, 0, c->stream>>>(static_cast<const float*>(d_in), w, n);
	auto transform = [&](double sign) {
		long long inner = 1;
		for (int a = 2; a >= 0; --a) {
			const int len = shape[a];
			const long long lines = (long long)n / len;
			if (len > 1) {
				const size_t smem = 2 * sizeof(double2) * size_t(len);
				dft_axis_kernel<<<unsigned(lines), kAcThreads, smem, c->stream>>>(w, len, inner, sign);
				c->launches += 1;
			}
			inner *= len;
		}
	};
	transform(-1.0);
	power_kernel<<<g, kAcThreads, 0, c->stream>>>(w, n);
	transform(+1.0);
	real_scaled_kernel<<<g, kAcThreads, 0, c->stream>>>(w, d_out, n, double(n));
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 3;
}

}  // namespace armab
