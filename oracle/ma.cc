/*
 * CPU oracle: the moving-average model -- TEST INFRASTRUCTURE ONLY.
 *
 * orc_ma_fit restates the fixed-point iteration of
 * MA_coefficient_solver::solve_fixed_point_iteration
 * (src/generator/ma_coefficient_solver.cc:36-139) with the solver's default
 * limits (src/generator/ma_coefficient_solver.hh:27-40) and
 * MA_white_noise_variance (src/arma.cc:73-79).
 *
 * orc_ma_filter restates the direct MA sum of the reference's convolution
 * test (src/test/convolution-test.cc:17-50): for every point, a running FP64
 * sum over k, i, j (ascending, bounded by the point's own indices) of
 * kernel(k,i,j) eps(t-k, x-i, y-j) with kernel = theta, kernel(0,0,0) = 0,
 * and zeta = eps - sum.  The reference's production path computes the same
 * linear convolution by FFT overlap-add (src/apmath/convolution.hh:58-130);
 * oracle/__init__.py restates that form with numpy for the comparison the
 * reference's test makes (tolerance 1e-4 there).
 */
#include <cmath>
#include <cstddef>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

inline size_t at3(int n1, int n2, int i, int j, int k) {
	return (size_t(i) * n1 + j) * n2 + k;
}

}  // namespace

extern "C" {

int orc_ma_fit(const double* acf, int at, int ax, int ay, int pt, int px, int py,
               double* theta, double* var_wn, int* iterations) {
	if (pt < 1 || px < 1 || py < 1 || pt > at || px > ax || py > ay) return 1;
	const int max_iterations = 1000;
	const double max_residual = 1e-5, min_var = 1e-6, eps_var = 1e-5;
	const size_t P = size_t(pt) * px * py;
	for (size_t q = 0; q < P; ++q) theta[q] = 0.0;
	double var = acf[0], old_var = 0.0, residual = 0.0;
	int it = 0;
	do {
		theta[0] = 0.0;
		for (int i = pt - 1; i >= 0; --i)
			for (int j = px - 1; j >= 0; --j)
				for (int k = py - 1; k >= 0; --k) {
					// sum over the box [ijk, order) x [0, order - ijk), row-major
					double s = 0.0;
					for (int l = i; l < pt; ++l)
						for (int m = j; m < px; ++m)
							for (int n = k; n < py; ++n)
								s += theta[at3(px, py, l, m, n)] *
								     theta[at3(px, py, l - i, m - j, n - k)];
					theta[at3(px, py, i, j, k)] = -acf[at3(ax, ay, i, j, k)] / var + s;
				}
		theta[0] = -1.0;
		for (size_t q = 0; q < P; ++q)
			if (!std::isfinite(theta[q])) return 2;
		residual = std::numeric_limits<double>::min();
		for (int i = 0; i < pt; ++i)
			for (int j = 0; j < px; ++j)
				for (int k = 0; k < py; ++k) {
					double s = 0.0;
					for (int l = i; l < pt; ++l)
						for (int m = j; m < px; ++m)
							for (int n = k; n < py; ++n)
								s += theta[at3(px, py, l, m, n)] *
								     theta[at3(px, py, l - i, m - j, n - k)];
					const double r = std::fabs(acf[at3(ax, ay, i, j, k)] - s * var);
					if (residual < r) residual = r;
				}
		old_var = var;
		double ss = 0.0;
		for (size_t q = 0; q < P; ++q) ss += theta[q] * theta[q];
		var = acf[0] / ss;
		if (var <= min_var) {
			*var_wn = var;
			return 3;
		}
		++it;
	} while (it < max_iterations && std::fabs(var - old_var) > eps_var && residual > max_residual);
	*var_wn = var;
	*iterations = it;
	return 0;
}

void orc_ma_filter(const double* theta, int pt, int px, int py, const double* eps, int nt,
                   int nx, int ny, double* zeta) {
	for (int t = 0; t < nt; ++t)
		for (int x = 0; x < nx; ++x)
			for (int y = 0; y < ny; ++y) {
				const int m1 = t + 1 < pt ? t + 1 : pt;
				const int m2 = x + 1 < px ? x + 1 : px;
				const int m3 = y + 1 < py ? y + 1 : py;
				double sum = 0.0;
				for (int k = 0; k < m1; ++k)
					for (int i = 0; i < m2; ++i)
						for (int j = 0; j < m3; ++j) {
							const double kern = (k | i | j) ? theta[at3(px, py, k, i, j)] : 0.0;
							sum += kern * eps[at3(nx, ny, t - k, x - i, y - j)];
						}
				zeta[at3(nx, ny, t, x, y)] = eps[at3(nx, ny, t, x, y)] - sum;
			}
}

}  // extern "C"
