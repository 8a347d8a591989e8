// Oracle (test infrastructure): the nonlinear inertialess transform (NIT) by
// per-point bisection on the target CDF.
#include "oracle.h"

#include <omp.h>

#include <cmath>

namespace {

constexpr double kPi = 3.14159265358979323846;
// Reference: src/physical_constants.hh:21-24 (truncated decimal literals).
constexpr double kSqrt2Pi = 2.506628274631;
constexpr double kSqrt2 = 1.4142135623731;

// 20-point Gauss-Legendre rule, positive half (10 nodes on (0,1) with their
// weights), computed here by Newton iteration on P_20.  The reference's Owen T
// (src/apmath/owen_t.cc:5-56) integrates the even integrand on [0,1] with the
// same rule, from a table of decimal literals.
struct GaussLegendre20 {
	double x[10], w[10];
	GaussLegendre20() {
		const int n = 20;
		for (int i = 0; i < 10; ++i) {
			// roots in decreasing order; index so that x[] ascends
			double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
			double pp = 0;
			for (int it = 0; it < 100; ++it) {
				double p1 = 1, p2 = 0;
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
			x[9 - i] = z;
			w[9 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
		}
	}
};

const GaussLegendre20& gl20() {
	static const GaussLegendre20 g;
	return g;
}

// Reference: src/linalg.hh:199-213 (bisection) as wrapped by
// linalg::Bisection (src/linalg.hh:220-268).  Stops when max_iter is reached,
// or the bracket is no wider than eps, or |f(c)| <= eps.
template <class F>
double bisection(double a, double b, F f, double eps, int max_iter) {
	double c, fc;
	int i = 0;
	do {
		c = 0.5 * (a + b);
		fc = f(c);
		if (f(a) * fc < 0.0) b = c;
		if (f(b) * fc < 0.0) a = c;
		i++;
	} while (i < max_iter && (b - a) > eps && std::fabs(fc) > eps);
	return c;
}

}  // namespace

// gsl_cdf_gaussian_P(x - mean, sigma) (src/stats/gaussian.hh:40-43), written
// through erfc.
extern "C" double orc_gaussian_cdf(double x, double mean, double sigma) {
	return 0.5 * std::erfc(-(x - mean) / (sigma * 1.41421356237309504880));
}

// Reference: src/apmath/owen_t.cc:34-56.
extern "C" double orc_owen_t(double h, double a) {
	const GaussLegendre20& g = gl20();
	double result = 0;
	const double a2 = a * a;
	const double h2 = -0.5 * h * h;
	for (int i = 0; i < 10; ++i) {
		const double x = g.x[i];
		const double term = (1.0 + a2 * x * x);
		result += g.w[i] * std::exp(h2 * term) / term;
	}
	return result * a / (2.0 * kPi);
}

// Reference: src/stats/skew_normal.hh:40-45, with the Gaussian member built
// from (mean, sigma) as the explicit constructor does.
extern "C" double orc_skew_normal_cdf(double x, double mean, double sigma,
                                      double alpha) {
	return orc_gaussian_cdf(x, mean, sigma) - 2.0 * orc_owen_t((x - mean) / sigma, alpha);
}

// Reference: src/stats/gram_charlier.hh:38-44 (kurtosis is non-excess).
extern "C" double orc_gram_charlier_cdf(double x, double s, double k) {
	return std::exp(-0.5 * x * x) *
	           (k * (3.0 * x - x * x * x) + s * (4.0 - 4.0 * x * x) +
	            3.0 * x * x * x - 9.0 * x) /
	           (24.0 * kSqrt2Pi) +
	       0.5 * std::erf(x / kSqrt2) + 0.5;
}

// Reference: src/nonlinear/nit_transform.cc:147-168 and
// src/nonlinear/transforms.hh:58-75.  Each value z is replaced by the root y
// of F_target(y) = Phi_sigma(z), sigma = sqrt(acf(0,0,0)).
extern "C" void orc_nit_transform(double* data, size_t n, double stdev, int kind,
                                  const double params[3], double a, double b,
                                  double eps, int max_iter, int nthreads) {
	if (nthreads <= 0) nthreads = omp_get_max_threads();
	const double p0 = params[0], p1 = params[1], p2 = params[2];
#pragma omp parallel for num_threads(nthreads) schedule(static)
	for (long long i = 0; i < (long long)n; ++i) {
		const double target = orc_gaussian_cdf(data[i], 0.0, stdev);
		if (kind == 0) {
			data[i] = bisection(a, b, [&](double x) {
				return orc_gram_charlier_cdf(x, p0, p1) - target;
			}, eps, max_iter);
		} else {
			data[i] = bisection(a, b, [&](double x) {
				return orc_skew_normal_cdf(x, p0, p1, p2) - target;
			}, eps, max_iter);
		}
	}
}
