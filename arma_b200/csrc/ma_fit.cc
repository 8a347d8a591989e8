// Moving-average coefficients by fixed-point iteration, the reference's MA
// fitting algorithm.
//
// Reference: MA_coefficient_solver::solve_fixed_point_iteration
// (src/generator/ma_coefficient_solver.cc:36-139, defaults in
// src/generator/ma_coefficient_solver.hh:27-40) and MA_white_noise_variance
// (src/arma.cc:73-79).  One sweep updates theta from the last lag to the
// first, in place (each update sees the lags already updated in the same
// sweep), with theta(0,0,0) held at 0:
//
//     theta(ijk) = -acf(ijk) / var_wn + sum_l theta(ijk + l) theta(l),
//
// l over the box [0, order - ijk).  Then theta(0,0,0) := -1, the residual
// max |acf(ijk) - var_wn sum_l theta(ijk + l) theta(l)| is taken, and
// var_wn := acf(0,0,0) / sum theta^2.  The loop ends after max_iterations
// sweeps, or once var_wn changes by at most eps, or once the residual is at
// most max_residual.  FP64 throughout, sums in row-major order of l.
#include <cmath>
#include <limits>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

// sum over l in [0, order - ijk) of theta(ijk + l) * theta(l), row-major in l
double lag_product(const std::vector<double>& th, const int o[3], int i, int j, int k) {
	double s = 0.0;
	for (int a = 0; a < o[0] - i; ++a)
		for (int b = 0; b < o[1] - j; ++b) {
			const double* hi = &th[(size_t(i + a) * o[1] + (j + b)) * o[2] + k];
			const double* lo = &th[(size_t(a) * o[1] + b) * o[2]];
			for (int c = 0; c < o[2] - k; ++c) s += hi[c] * lo[c];
		}
	return s;
}

}  // namespace

double ma_white_noise_variance(const double* acf, const double* theta, const int order[3]) {
	const size_t P = size_t(order[0]) * order[1] * order[2];
	double s = 0.0;
	for (size_t q = 0; q < P; ++q) s += theta[q] * theta[q];
	return acf[0] / s;
}

int ma_fit_fixed_point(const double* acf, const int acf_shape[3], const int order[3],
                       const MaFitOptions& opt, std::vector<double>* theta_out, double* var_out,
                       int* iterations, double* residual_out) {
	for (int a = 0; a < 3; ++a)
		if (order[a] <= 0 || order[a] > acf_shape[a]) return 1;
	const int o[3] = {order[0], order[1], order[2]};
	const size_t P = size_t(o[0]) * o[1] * o[2];
	// the ACF restricted to the order's box (the solver indexes acf(ijk) with
	// ijk < order)
	std::vector<double> g(P);
	for (int i = 0; i < o[0]; ++i)
		for (int j = 0; j < o[1]; ++j)
			for (int k = 0; k < o[2]; ++k)
				g[(size_t(i) * o[1] + j) * o[2] + k] =
				    acf[(size_t(i) * acf_shape[1] + j) * acf_shape[2] + k];
	std::vector<double> th(P, 0.0);
	double var = g[0], old_var = 0.0, residual = 0.0;
	int it = 0;
	do {
		th[0] = 0.0;
		for (int i = o[0] - 1; i >= 0; --i)
			for (int j = o[1] - 1; j >= 0; --j)
				for (int k = o[2] - 1; k >= 0; --k) {
					const size_t q = (size_t(i) * o[1] + j) * o[2] + k;
					th[q] = -g[q] / var + lag_product(th, o, i, j, k);
				}
		th[0] = -1.0;
		for (double v : th)
			if (!std::isfinite(v)) return 2;
		residual = std::numeric_limits<double>::min();
		for (int i = 0; i < o[0]; ++i)
			for (int j = 0; j < o[1]; ++j)
				for (int k = 0; k < o[2]; ++k) {
					const size_t q = (size_t(i) * o[1] + j) * o[2] + k;
					const double r = std::fabs(g[q] - lag_product(th, o, i, j, k) * var);
					if (residual < r) residual = r;
				}
		old_var = var;
		var = ma_white_noise_variance(g.data(), th.data(), o);
		if (var <= opt.min_var_wn) {
			if (var_out) *var_out = var;
			return 3;
		}
		++it;
	} while (it < opt.max_iterations && std::fabs(var - old_var) > opt.eps &&
	         residual > opt.max_residual);
	*theta_out = std::move(th);
	if (var_out) *var_out = var;
	if (iterations) *iterations = it;
	if (residual_out) *residual_out = residual;
	return 0;
}

}  // namespace armab
