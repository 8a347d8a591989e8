// Target distributions of the nonlinear inertialess transform, usable on the
// host and the device.
//
//   Gaussian CDF      gsl_cdf_gaussian_P(x - mean, sigma)
//                     (reference src/stats/gaussian.hh:40-43), via erfc.
//   Gram-Charlier CDF (reference src/stats/gram_charlier.hh:38-44): kurtosis is
//                     the non-excess fourth standardised moment.
//   Skew-normal CDF   Phi_{mean,sigma}(x) - 2 T((x-mean)/sigma, alpha)
//                     (reference src/stats/skew_normal.hh:40-45).
//   Owen's T          (reference src/apmath/owen_t.cc:34-56): the even
//                     integrand on [0,1] by the positive half of the 20-point
//                     Gauss-Legendre rule.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define ARMA_HD __host__ __device__ __forceinline__
#else
#define ARMA_HD inline
#endif

namespace armab {
namespace dist {

// Constants used by the reference's distribution code
// (src/physical_constants.hh:21-24 truncates sqrt(2*pi) and sqrt(2)).
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt2PiRef = 2.506628274631;
constexpr double kSqrt2Ref = 1.4142135623731;

// Nodes and weights of the 20-point Gauss-Legendre rule on (0,1), ascending.
struct GL20 {
	double x[10];
	double w[10];
};

// Computed by Newton's method on the Legendre polynomial P_20 (host).
inline GL20 make_gl20() {
	GL20 g{};
	const int n = 20;
	for (int i = 0; i < 10; ++i) {
		double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
		double pp = 0.0;
		for (int it = 0; it < 100; ++it) {
			double p1 = 1.0, p2 = 0.0;
			for (int j = 1; j <= n; ++j) {
				const double p3 = p2;
				p2 = p1;
				p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
			}
			pp = n * (z * p1 - p2) / (z * z - 1.0);
			const double z1 = z;
			z = z1 - p1 / pp;
			if (std::fabs(z - z1) < 1e-16) break;
		}
		g.x[9 - i] = z;
		g.w[9 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
	}
	return g;
}

inline const GL20& gl20_host() {
	static const GL20 g = make_gl20();
	return g;
}

ARMA_HD double gaussian_cdf(double x, double mean, double sigma) {
	return 0.5 * erfc(-(x - mean) / (sigma * 1.41421356237309504880));
}

ARMA_HD double owen_t(double h, double a, const GL20& g) {
	double result = 0.0;
	const double a2 = a * a;
	const double h2 = -0.5 * h * h;
	for (int i = 0; i < 10; ++i) {
		const double x = g.x[i];
		const double term = 1.0 + a2 * x * x;
		result += g.w[i] * exp(h2 * term) / term;
	}
	return result * a / (2.0 * kPi);
}

ARMA_HD double skew_normal_cdf(double x, double mean, double sigma, double alpha,
                               const GL20& g) {
	return gaussian_cdf(x, mean, sigma) - 2.0 * owen_t((x - mean) / sigma, alpha, g);
}

ARMA_HD double gram_charlier_cdf(double x, double s, double k) {
	return exp(-0.5 * x * x) *
	           (k * (3.0 * x - x * x * x) + s * (4.0 - 4.0 * x * x) + 3.0 * x * x * x -
	            9.0 * x) /
	           (24.0 * kSqrt2PiRef) +
	       0.5 * erf(x / kSqrt2Ref) + 0.5;
}

// dist 0 = Gram-Charlier {skewness, kurtosis}; 1 = skew normal {mean, stdev, alpha}.
ARMA_HD double target_cdf(int d, const double* p, double x, const GL20& g) {
	return d == 0 ? gram_charlier_cdf(x, p[0], p[1]) : skew_normal_cdf(x, p[0], p[1], p[2], g);
}

inline double target_cdf(int d, const double* p, double x) {
	return target_cdf(d, p, x, gl20_host());
}

}  // namespace dist
}  // namespace armab
