// The empirical ACF of a wave group: what the reference's AR model reads under
// `acf = { func = cos|sin|stokes|standing_wave ... nwaves ... shape ... }`.
//
// Reference: ACF_generator::generate and its helpers
// (src/generator/acf_generator.cc:132-244, src/generator/acf_generator.hh:
// 30-45, 150-175), the plain-wave profiles (src/generator/plain_wave.hh:40-120,
// names in src/generator/plain_wave_profile.cc:7-22) and auto_covariance
// (src/arma.cc:81-100).  A plain wave is sampled on the domain [-nwaves,
// nwaves] per axis with 2 shape + 1 points (or, when a shape component is 0,
// on doubling sizes from 3 points until the variance changes by less than
// 1e-3, below 64), multiplied by exp(-(alpha_t |t| + alpha_x |x| + alpha_y
// |y|)) and rescaled to the wave's variance; the ACF is the circular
// auto-covariance IFFT(|FFT(w)|^2) / n^2 truncated to half of each axis, on a
// grid of length nwaves per axis.  FP64 on the host; the 3-D transforms are
// mixed-radix FFTs along each axis (any length; a prime factor p costs p
// operations per value and level).
#include <cmath>
#include <complex>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double k2Pi = 2.0 * kPi;

double plain_wave(const EmpiricalAcf& p, double x, double y, double t) {
	const double kx = p.wavenum[0], ky = p.wavenum[1], v = p.velocity, a = p.amplitude;
	switch (p.func) {
		case 0:  // sin
			return a * std::sin(k2Pi * (kx * x + ky * y - v * t));
		case 1:  // cos = sin with phase pi/2
			return a * std::sin(k2Pi * (kx * x + ky * y - v * t) + 0.5 * kPi);
		case 2: {  // stokes
			const double theta = k2Pi * (kx * x + ky * y - v * t);
			const double steep = k2Pi * a * std::sqrt(kx * kx + ky * ky);
			return a * (std::cos(theta) + 0.5 * steep * std::cos(2.0 * theta) +
			            (3.0 / 8.0) * steep * steep * std::cos(3.0 * theta));
		}
		default:  // standing wave
			return a * std::cos(k2Pi * (kx * x + ky * y)) * std::cos(k2Pi * (v * t));
	}
}

// Unbiased variance with a running mean, as gsl_stats_variance.
double variance(const std::vector<double>& w) {
	long double mean = 0.0L;
	for (size_t i = 0; i < w.size(); ++i) mean += (w[i] - mean) / (long double)(i + 1);
	long double s = 0.0L;
	for (double v : w) {
		const long double d = v - mean;
		s += d * d;
	}
	return double(s / (long double)(w.size() - 1));
}

// The wave sampled on [-nwaves, nwaves] with n points per axis.
std::vector<double> sample(const EmpiricalAcf& p, const int n[3]) {
	std::vector<double> w(size_t(n[0]) * n[1] * n[2]);
	double d[3];
	for (int a = 0; a < 3; ++a) d[a] = 2.0 * p.nwaves[a] / std::max(n[a] - 1, 1);
	for (int i = 0; i < n[0]; ++i)
		for (int j = 0; j < n[1]; ++j)
			for (int k = 0; k < n[2]; ++k) {
				const double t = -p.nwaves[0] + d[0] * i;
				const double x = -p.nwaves[1] + d[1] * j;
				const double y = -p.nwaves[2] + d[2] * k;
				w[(size_t(i) * n[1] + j) * n[2] + k] = plain_wave(p, x, y, t);
			}
	return w;
}

// Unnormalised mixed-radix DFT of x[0], x[stride], ... (n values) into
// out[0..n): decimation in time by the smallest prime factor p of n, each
// output combined directly from the p sub-transforms (n p operations per
// level).  tw[j] = exp(sign 2 pi i j / N) for the full length N; `step` = N / n.
void fft_rec(const std::complex<double>* x, size_t stride, int n, std::complex<double>* out,
             std::complex<double>* tmp, const std::vector<std::complex<double>>& tw, int step) {
	if (n == 1) {
		out[0] = x[0];
		return;
	}
	int p = 2;
	while (n % p) p = p * p > n ? n : p + 1;
	const int m = n / p;
	for (int r = 0; r < p; ++r) fft_rec(x + r * stride, stride * p, m, tmp + r * m, out, tw, step * p);
	const int big = int(tw.size());
	for (int k = 0; k < m; ++k)
		for (int q = 0; q < p; ++q) {
			const int kk = q * m + k;
			std::complex<double> acc = tmp[k];
			for (int r = 1; r < p; ++r)
				acc += tmp[r * m + k] * tw[(size_t(r) * kk % n) * step % big];
			out[kk] = acc;
		}
}

// Unnormalised DFT along one axis of an n0 x n1 x n2 complex array.
void dft_axis(std::vector<std::complex<double>>& a, const int n[3], int axis, int sign) {
	const int len = n[axis];
	std::vector<std::complex<double>> tw(len), in(len), out(len), tmp(len);
	for (int k = 0; k < len; ++k) tw[k] = std::polar(1.0, sign * k2Pi * k / len);
	const size_t stride = axis == 0 ? size_t(n[1]) * n[2] : axis == 1 ? size_t(n[2]) : 1;
	const int o1 = axis == 0 ? n[1] : n[0], o2 = axis == 2 ? n[1] : n[2];
	for (int u = 0; u < o1; ++u)
		for (int v = 0; v < o2; ++v) {
			size_t base;
			if (axis == 0) base = size_t(u) * n[2] + v;
			else if (axis == 1) base = size_t(u) * n[1] * n[2] + v;
			else base = (size_t(u) * n[1] + v) * n[2];
			for (int q = 0; q < len; ++q) in[q] = a[base + q * stride];
			fft_rec(in.data(), 1, len, out.data(), tmp.data(), tw, 1);
			for (int q = 0; q < len; ++q) a[base + q * stride] = out[q];
		}
}

}  // namespace

std::vector<double> empirical_acf(const EmpiricalAcf& p, int shape[3], double delta[3]) {
	int n[3];
	std::vector<double> w;
	if (p.shape[0] > 0 && p.shape[1] > 0 && p.shape[2] > 0) {
		for (int a = 0; a < 3; ++a) n[a] = 2 * p.shape[a] + 1;
		w = sample(p, n);
	} else {  // the smallest wave size whose variance has settled
		int ws[3] = {2, 2, 2};
		double var = -1.0, var0;
		while (ws[0] < 64 && ws[1] < 64 && ws[2] < 64) {
			for (int a = 0; a < 3; ++a) n[a] = ws[a] + 1;
			w = sample(p, n);
			var0 = var;
			var = variance(w);
			if (!(var0 < 0.0) && std::fabs(var - var0) < 1e-3) break;
			for (int a = 0; a < 3; ++a) ws[a] *= 2;
		}
	}
	// exponential decay, rescaled to the wave's variance
	const double v0 = variance(w);
	std::vector<double> we(w.size());
	double d[3];
	for (int a = 0; a < 3; ++a) d[a] = 2.0 * p.nwaves[a] / std::max(n[a] - 1, 1);
	for (int i = 0; i < n[0]; ++i)
		for (int j = 0; j < n[1]; ++j)
			for (int k = 0; k < n[2]; ++k) {
				const double t = -p.nwaves[0] + d[0] * i;
				const double x = -p.nwaves[1] + d[1] * j;
				const double y = -p.nwaves[2] + d[2] * k;
				const size_t q = (size_t(i) * n[1] + j) * n[2] + k;
				we[q] = w[q] * std::exp(-(std::fabs(t * p.alpha[0]) + std::fabs(x * p.alpha[1]) +
				                          std::fabs(y * p.alpha[2])));
			}
	const double sc = std::sqrt(v0 / variance(we));
	for (double& v : we) v *= sc;
	const std::vector<double> c = auto_covariance(we, n);
	for (int a = 0; a < 3; ++a) {
		shape[a] = n[a] / 2;
		delta[a] = p.nwaves[a] / std::max(shape[a] - 1, 1);  // Grid(shape, nwaves)
	}
	std::vector<double> acf(size_t(shape[0]) * shape[1] * shape[2]);
	for (int i = 0; i < shape[0]; ++i)
		for (int j = 0; j < shape[1]; ++j)
			for (int k = 0; k < shape[2]; ++k)
				acf[(size_t(i) * shape[1] + j) * shape[2] + k] = c[(size_t(i) * n[1] + j) * n[2] + k];
	return acf;
}

// Circular auto-covariance Re IFFT(|FFT(w)|^2) / n / n over the whole array
// (auto_covariance, src/arma.cc:81-100): element (i,j,k) is
// sum w(i1,j1,k1) w((i+i1)%n0, (j+j1)%n1, (k+k1)%n2) / n.
std::vector<double> auto_covariance(const std::vector<double>& w, const int n[3]) {
	std::vector<std::complex<double>> c(w.begin(), w.end());
	for (int a = 0; a < 3; ++a) dft_axis(c, n, a, -1);
	for (auto& v : c) v = std::norm(v);
	for (int a = 0; a < 3; ++a) dft_axis(c, n, a, +1);
	const double nn = double(c.size());
	std::vector<double> out(c.size());
	for (size_t q = 0; q < c.size(); ++q) out[q] = c[q].real() / nn / nn;
	return out;
}

}  // namespace armab
