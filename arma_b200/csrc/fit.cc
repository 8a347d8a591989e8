// Host FP64 model fitting: analytic ACF, Yule-Walker block-Toeplitz system,
// LL^T Cholesky solve, white-noise variance, the intra-slice impulse response
// used by the FP32 filter, and the NIT inverse-CDF table.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "distributions.h"
#include "internal.h"

namespace armab {
namespace {

// Blocked right-looking LL^T Cholesky factorisation followed by the two
// triangular solves; FP64 throughout.  A is n x n row-major (lower triangle
// used and overwritten).  Returns 0 or the 1-based index of the first
// non-positive pivot.
int cholesky_solve(int n, double* A, double* b) {
	auto a = [&](int i, int j) -> double& { return A[size_t(i) * n + j]; };
	const int nb = 64;
	for (int k0 = 0; k0 < n; k0 += nb) {
		const int k1 = std::min(n, k0 + nb);
		// factor the diagonal block and the panel below it
		for (int j = k0; j < k1; ++j) {
			double s = a(j, j);
			for (int k = k0; k < j; ++k) s -= a(j, k) * a(j, k);
			if (!(s > 0.0)) return j + 1;
			const double d = std::sqrt(s);
			a(j, j) = d;
			const double inv = 1.0 / d;
#pragma omp parallel for schedule(static) if (n - j > 256)
			for (int i = j + 1; i < n; ++i) {
				double t = a(i, j);
				for (int k = k0; k < j; ++k) t -= a(i, k) * a(j, k);
				a(i, j) = t * inv;
			}
		}
		// trailing update A22 -= L21 L21^T (lower triangle)
#pragma omp parallel for schedule(dynamic, 8) if (n - k1 > 128)
		for (int i = k1; i < n; ++i) {
			const double* li = &a(i, k0);
			for (int j = k1; j <= i; ++j) {
				const double* lj = &a(j, k0);
				double t = 0.0;
				for (int k = 0; k < k1 - k0; ++k) t += li[k] * lj[k];
				a(i, j) -= t;
			}
		}
	}
	for (int i = 0; i < n; ++i) {
		double t = b[i];
		for (int k = 0; k < i; ++k) t -= a(i, k) * b[k];
		b[i] = t / a(i, i);
	}
	for (int i = n - 1; i >= 0; --i) {
		double t = b[i];
		for (int k = i + 1; k < n; ++k) t -= a(k, i) * b[k];
		b[i] = t / a(i, i);
	}
	return 0;
}

double acf_value(int kind, double amp, double vel, const double* al, const double* be,
                 const double* dl, int i, int j, int k) {
	// gamma at a signed lag (i, j, k): the exponential uses |lag|; the cosine
	// factors are even per axis (standing) or jointly even (propagating).
	const double e = std::exp(-(al[0] * std::abs(i) * dl[0] + al[1] * std::abs(j) * dl[1] +
	                            al[2] * std::abs(k) * dl[2]));
	if (kind == ARMA_ACF_PROPAGATING)
		return amp * e * std::cos(vel * i * dl[0] + be[0] * j * dl[1] + be[1] * k * dl[2]);
	return amp * e * std::cos(vel * i * dl[0]) * std::cos(be[0] * j * dl[1]) *
	       std::cos(be[1] * k * dl[2]);
}

int solve_yw(std::vector<double>& R, int P, const double* acf, int ax, int ay,
             const int order[3], double* phi, double* var_wn) {
	const int m = P - 1;
	std::vector<double> lhs(size_t(m) * m), rhs(m);
	for (int i = 0; i < m; ++i) {
		rhs[i] = R[size_t(i + 1) * P];
		std::copy(&R[size_t(i + 1) * P + 1], &R[size_t(i + 1) * P + 1] + m, &lhs[size_t(i) * m]);
	}
	if (m > 0) {
		const int info = cholesky_solve(m, lhs.data(), rhs.data());
		if (info != 0) return info;
	}
	phi[0] = 0.0;
	std::copy(rhs.begin(), rhs.end(), phi + 1);
	// white_noise_variance: acf(0,0,0) - sum(phi * acf(order box)), C order
	double s = 0.0;
	for (int i = 0; i < order[0]; ++i)
		for (int j = 0; j < order[1]; ++j)
			for (int k = 0; k < order[2]; ++k)
				s += phi[(size_t(i) * order[1] + j) * order[2] + k] *
				     acf[(size_t(i) * ax + j) * ay + k];
	*var_wn = acf[0] - s;
	return 0;
}

}  // namespace

void acf_eval(int kind, double amplitude, double velocity, const double alpha[3],
              const double beta[2], const double delta[3], const int shape[3],
              double* out) {
	for (int i = 0; i < shape[0]; ++i)
		for (int j = 0; j < shape[1]; ++j)
			for (int k = 0; k < shape[2]; ++k)
				out[(size_t(i) * shape[1] + j) * shape[2] + k] =
				    acf_value(kind, amplitude, velocity, alpha, beta, delta, i, j, k);
}

int fit_gauss_table(const double* acf, const int acf_shape[3], const int order[3],
                    int method, double* phi, double* var_wn) {
	(void)method;
	const int pt = order[0], px = order[1], py = order[2];
	const int P = pt * px * py;
	const int ax = acf_shape[1], ay = acf_shape[2];
	std::vector<double> R(size_t(P) * P);
	for (int r = 0; r < P; ++r) {
		const int i = r / (px * py), i2 = (r / py) % px, i3 = r % py;
		for (int q = 0; q < P; ++q) {
			const int j = q / (px * py), j2 = (q / py) % px, j3 = q % py;
			R[size_t(r) * P + q] =
			    acf[(size_t(std::abs(i - j)) * ax + std::abs(i2 - j2)) * ay + std::abs(i3 - j3)];
		}
	}
	return solve_yw(R, P, acf, ax, ay, order, phi, var_wn);
}

int fit_analytic(int kind, double amplitude, double velocity, const double alpha[3],
                 const double beta[2], const double delta[3], const int order[3],
                 double* phi, double* var_wn) {
	const int pt = order[0], px = order[1], py = order[2];
	const int P = pt * px * py;
	std::vector<double> acf(static_cast<size_t>(P));
	acf_eval(kind, amplitude, velocity, alpha, beta, delta, order, acf.data());
	std::vector<double> R(size_t(P) * P);
	for (int r = 0; r < P; ++r) {
		const int i = r / (px * py), i2 = (r / py) % px, i3 = r % py;
		for (int q = 0; q < P; ++q) {
			const int j = q / (px * py), j2 = (q / py) % px, j3 = q % py;
			R[size_t(r) * P + q] =
			    acf_value(kind, amplitude, velocity, alpha, beta, delta, i - j, i2 - j2, i3 - j3);
		}
	}
	return solve_yw(R, P, acf.data(), px, py, order, phi, var_wn);
}

void intra_slice_response(const double* phi, const int order[3], int tx, int ty,
                          double* h) {
	const int px = order[1], py = order[2];
	for (int x = 0; x < tx; ++x)
		for (int y = 0; y < ty; ++y) {
			double s = (x == 0 && y == 0) ? 1.0 : 0.0;
			for (int i = 0; i < std::min(x + 1, px); ++i)
				for (int j = 0; j < std::min(y + 1, py); ++j) {
					if (i == 0 && j == 0) continue;
					s += phi[size_t(i) * py + j] * h[size_t(x - i) * ty + (y - j)];
				}
			h[size_t(x) * ty + y] = s;
		}
}

void nit_build_lut(int dist, const double params[3], double stdev, int nodes,
                   double range, double* x0, double* dx, std::vector<double>& y) {
	const double lo = -range * stdev, hi = range * stdev;
	*x0 = lo;
	*dx = (hi - lo) / (nodes - 1);
	y.resize(nodes);
#pragma omp parallel for schedule(static)
	for (int i = 0; i < nodes; ++i) {
		const double x = lo + *dx * i;
		const double target = dist::gaussian_cdf(x, 0.0, stdev);
		// bracket the root of F(y) - target, then bisect to full precision
		double a = -64.0, b = 64.0;
		auto f = [&](double v) { return dist::target_cdf(dist, params, v) - target; };
		double fa = f(a);
		for (int it = 0; it < 200 && (b - a) > 1e-15 * std::max(1.0, std::fabs(a)); ++it) {
			const double c = 0.5 * (a + b);
			const double fc = f(c);
			if ((fa < 0.0) == (fc < 0.0)) { a = c; fa = fc; } else { b = c; }
		}
		y[i] = 0.5 * (a + b);
	}
}

std::vector<double> nit_lut_coefficients(const std::vector<double>& y) {
	const int nodes = int(y.size());
	std::vector<double> c(4 * size_t(nodes + 1), 0.0);
	// Lagrange basis on the nodes s = -1, 0, 1, 2 (values y[i-1 .. i+2]) with
	// s = t + d: basis m is prod_{q != m} (t - e_q) / den_m, e_q = s_q - d.
	const int sq[4] = {-1, 0, 1, 2};
	const double den[4] = {-6.0, 2.0, -2.0, 6.0};
	for (int j = 0; j + 1 < nodes; ++j) {
		const int i = std::min(std::max(j, 1), nodes - 3);
		const int d = j - i;
		double* out = &c[4 * size_t(j)];
		for (int m = 0; m < 4; ++m) {
			double e[3];
			int r = 0;
			for (int q = 0; q < 4; ++q)
				if (q != m) e[r++] = double(sq[q] - d);
			// (t - a)(t - b)(t - c) = t^3 - (a+b+c) t^2 + (ab+bc+ca) t - abc
			const double w = y[size_t(i - 1 + m)] / den[m];
			out[0] += -e[0] * e[1] * e[2] * w;
			out[1] += (e[0] * e[1] + e[1] * e[2] + e[2] * e[0]) * w;
			out[2] += -(e[0] + e[1] + e[2]) * w;
			out[3] += w;
		}
	}
	double* lo = &c[4 * size_t(nodes - 1)];
	lo[0] = y[0];
	lo[1] = y[1] - y[0];
	double* hi = &c[4 * size_t(nodes)];
	hi[0] = y[size_t(nodes - 1)];
	hi[1] = y[size_t(nodes - 1)] - y[size_t(nodes - 2)];
	return c;
}

}  // namespace armab
