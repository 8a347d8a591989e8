// Oracle (test infrastructure): analytic ACF, block-Toeplitz YW matrix,
// symmetric solves and the Gauss-elimination AR fit.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

// Reference: src/acf.hh:18-62.  The blitz expression is evaluated per lag
// point in the same operand order: amplitude * exp(-(a0*i*d0 + a1*j*d1 +
// a2*k*d2)) * cos(...) ...
template <bool Propagating>
void acf_fill(double amp, double vel, const double* alpha, const double* beta,
              const double* delta, int nt, int nx, int ny, double* out) {
	for (int i = 0; i < nt; ++i) {
		for (int j = 0; j < nx; ++j) {
			for (int k = 0; k < ny; ++k) {
				const double e = std::exp(-(alpha[0] * i * delta[0] +
				                            alpha[1] * j * delta[1] +
				                            alpha[2] * k * delta[2]));
				double v;
				if (Propagating) {
					v = amp * e *
					    std::cos(vel * i * delta[0] + beta[0] * j * delta[1] +
					             beta[1] * k * delta[2]);
				} else {
					v = amp * e * std::cos(vel * i * delta[0]) *
					    std::cos(beta[0] * j * delta[1]) *
					    std::cos(beta[1] * k * delta[2]);
				}
				out[(size_t(i) * nx + j) * ny + k] = v;
			}
		}
	}
}

}  // namespace

extern "C" void orc_acf_standing(double amplitude, double velocity,
                                 const double alpha[3], const double beta[2],
                                 const double delta[3], int nt, int nx, int ny,
                                 double* out) {
	acf_fill<false>(amplitude, velocity, alpha, beta, delta, nt, nx, ny, out);
}

extern "C" void orc_acf_propagating(double amplitude, double velocity,
                                    const double alpha[3], const double beta[2],
                                    const double delta[3], int nt, int nx,
                                    int ny, double* out) {
	acf_fill<true>(amplitude, velocity, alpha, beta, delta, nt, nx, ny, out);
}

// Reference: src/generator/voodoo.cc:58-104.  R[(t,x,y),(t',x',y')] =
// acf(|t-t'|, |x-x'|, |y-y'|): three nested levels of symmetric Toeplitz
// blocks; rows and columns are flattened in C order of the order box.
extern "C" void orc_ac_matrix(const double* acf, int at, int ax, int ay, int pt,
                              int px, int py, double* out) {
	(void)at;
	const int P = pt * px * py;
	for (int i = 0; i < pt; ++i)
		for (int i2 = 0; i2 < px; ++i2)
			for (int i3 = 0; i3 < py; ++i3) {
				const int r = (i * px + i2) * py + i3;
				for (int j = 0; j < pt; ++j)
					for (int j2 = 0; j2 < px; ++j2)
						for (int j3 = 0; j3 < py; ++j3) {
							const int c = (j * px + j2) * py + j3;
							const int a = std::abs(i - j), b = std::abs(i2 - j2),
							          d = std::abs(i3 - j3);
							out[size_t(r) * P + c] = acf[(size_t(a) * ax + b) * ay + d];
						}
			}
}

// Symmetric-indefinite solve with the upper triangle (reference
// src/linalg.cc:22-35 calls LAPACKE_dsysv('U')).  This is the unblocked
// Bunch-Kaufman diagonal pivoting method (LAPACK dsytf2 'U', alpha =
// (1+sqrt(17))/8, factorisation A = U D U^T proceeding from the last column)
// followed by the matching triangular solves.  The blocked LAPACK routine
// makes the same pivot choices in exact arithmetic; rounding may differ.
extern "C" int orc_sysv_upper(int n, double* A, double* b) {
	auto a = [&](int i, int j) -> double& { return A[size_t(i) * n + j]; };
	// Work only with the upper triangle: a(i,j) for i <= j.
	const double alpha = (1.0 + std::sqrt(17.0)) / 8.0;
	std::vector<int> ipiv(n);
	int k = n - 1;
	while (k >= 0) {
		int kstep = 1;
		const double absakk = std::fabs(a(k, k));
		int imax = 0;
		double colmax = 0.0;
		if (k > 0) {
			for (int i = 0; i < k; ++i)
				if (std::fabs(a(i, k)) > colmax) { colmax = std::fabs(a(i, k)); imax = i; }
		}
		int kp;
		if (std::max(absakk, colmax) == 0.0) return k + 1;  // singular
		if (absakk >= alpha * colmax) {
			kp = k;
		} else {
			double rowmax = 0.0;
			for (int j = imax + 1; j <= k; ++j) rowmax = std::max(rowmax, std::fabs(a(imax, j)));
			for (int j = 0; j < imax; ++j) rowmax = std::max(rowmax, std::fabs(a(j, imax)));
			if (absakk >= alpha * colmax * (colmax / rowmax)) {
				kp = k;
			} else if (std::fabs(a(imax, imax)) >= alpha * rowmax) {
				kp = imax;
			} else {
				kp = imax;
				kstep = 2;
			}
		}
		const int kk = k - kstep + 1;
		if (kp != kk) {
			// interchange rows/columns kk and kp in the leading submatrix
			for (int i = 0; i < kp; ++i) std::swap(a(i, kk), a(i, kp));
			for (int j = kp + 1; j < kk; ++j) std::swap(a(j, kk), a(kp, j));
			std::swap(a(kk, kk), a(kp, kp));
			if (kstep == 2) std::swap(a(k - 1, k), a(kp, k));
		}
		if (kstep == 1) {
			const double r1 = 1.0 / a(k, k);
			// rank-1 update of the leading k x k block (upper part)
			for (int j = 0; j < k; ++j) {
				const double t = -r1 * a(j, k);
				for (int i = 0; i <= j; ++i) a(i, j) += t * a(i, k);
			}
			for (int i = 0; i < k; ++i) a(i, k) *= r1;
		} else if (k > 1) {
			double d12 = a(k - 1, k);
			const double d22 = a(k - 1, k - 1) / d12;
			const double d11 = a(k, k) / d12;
			const double t = 1.0 / (d11 * d22 - 1.0);
			d12 = t / d12;
			for (int j = k - 2; j >= 0; --j) {
				const double wkm1 = d12 * (d11 * a(j, k - 1) - a(j, k));
				const double wk = d12 * (d22 * a(j, k) - a(j, k - 1));
				for (int i = j; i >= 0; --i)
					a(i, j) = a(i, j) - a(i, k) * wk - a(i, k - 1) * wkm1;
				a(j, k) = wk;
				a(j, k - 1) = wkm1;
			}
		}
		if (kstep == 1) {
			ipiv[k] = kp;
		} else {
			ipiv[k] = -(kp + 1);
			ipiv[k - 1] = -(kp + 1);
		}
		k -= kstep;
	}
	// Solve U D U^T x = b (LAPACK dsytrs 'U').
	k = n - 1;
	while (k >= 0) {
		if (ipiv[k] >= 0) {
			const int kp = ipiv[k];
			if (kp != k) std::swap(b[k], b[kp]);
			for (int i = 0; i < k; ++i) b[i] -= a(i, k) * b[k];
			b[k] *= 1.0 / a(k, k);
			k -= 1;
		} else {
			const int kp = -ipiv[k] - 1;
			if (kp != k - 1) std::swap(b[k - 1], b[kp]);
			for (int i = 0; i < k - 1; ++i) {
				b[i] -= a(i, k) * b[k];
				b[i] -= a(i, k - 1) * b[k - 1];
			}
			const double akm1k = a(k - 1, k);
			const double akm1 = a(k - 1, k - 1) / akm1k;
			const double ak = a(k, k) / akm1k;
			const double denom = akm1 * ak - 1.0;
			const double bkm1 = b[k - 1] / akm1k;
			const double bk = b[k] / akm1k;
			b[k - 1] = (ak * bkm1 - bk) / denom;
			b[k] = (akm1 * bk - bkm1) / denom;
			k -= 2;
		}
	}
	k = 0;
	while (k < n) {
		if (ipiv[k] >= 0) {
			double t = 0.0;
			for (int i = 0; i < k; ++i) t += a(i, k) * b[i];
			b[k] -= t;
			const int kp = ipiv[k];
			if (kp != k) std::swap(b[k], b[kp]);
			k += 1;
		} else {
			double t0 = 0.0, t1 = 0.0;
			for (int i = 0; i < k; ++i) {
				t0 += a(i, k) * b[i];
				t1 += a(i, k + 1) * b[i];
			}
			b[k] -= t0;
			b[k + 1] -= t1;
			const int kp = -ipiv[k] - 1;
			if (kp != k) std::swap(b[k], b[kp]);
			k += 2;
		}
	}
	return 0;
}

// Dense LL^T Cholesky solve (lower factor), FP64.
extern "C" int orc_cholesky_solve(int n, double* A, double* b) {
	auto a = [&](int i, int j) -> double& { return A[size_t(i) * n + j]; };
	for (int j = 0; j < n; ++j) {
		double s = a(j, j);
		for (int k = 0; k < j; ++k) s -= a(j, k) * a(j, k);
		if (!(s > 0.0)) return j + 1;
		const double d = std::sqrt(s);
		a(j, j) = d;
		for (int i = j + 1; i < n; ++i) {
			double t = a(i, j);
			for (int k = 0; k < j; ++k) t -= a(i, k) * a(j, k);
			a(i, j) = t / d;
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

// Reference: src/generator/ar_model.cc:55-61.  var_wn = acf(0,0,0) -
// sum(phi * acf(order box)); the blitz reduction runs in C order.
extern "C" double orc_white_noise_variance(const double* acf, int at, int ax,
                                           int ay, const double* phi, int pt,
                                           int px, int py) {
	(void)at;
	double s = 0.0;
	for (int i = 0; i < pt; ++i)
		for (int j = 0; j < px; ++j)
			for (int k = 0; k < py; ++k)
				s += phi[(size_t(i) * px + j) * py + k] * acf[(size_t(i) * ax + j) * ay + k];
	return acf[0] - s;
}

// Reference: src/generator/ar_model.cc:97-135.  Drop the first row/column of
// the auto-covariance matrix, move its first column to the right-hand side,
// solve, and set phi(0,0,0) = 0.
extern "C" int orc_ar_fit_gauss(const double* acf, int at, int ax, int ay,
                                int pt, int px, int py, int method, double* phi,
                                double* var_wn) {
	if (pt > at || px > ax || py > ay) return -1;
	const int P = pt * px * py;
	std::vector<double> R(size_t(P) * P);
	orc_ac_matrix(acf, at, ax, ay, pt, px, py, R.data());
	const int m = P - 1;
	std::vector<double> lhs(size_t(m) * m), rhs(m);
	for (int i = 0; i < m; ++i) {
		rhs[i] = R[size_t(i + 1) * P + 0];
		for (int j = 0; j < m; ++j) lhs[size_t(i) * m + j] = R[size_t(i + 1) * P + j + 1];
	}
	int info = (method == 0) ? orc_sysv_upper(m, lhs.data(), rhs.data())
	                         : orc_cholesky_solve(m, lhs.data(), rhs.data());
	if (info != 0) return info;
	phi[0] = 0.0;
	std::copy(rhs.begin(), rhs.end(), phi + 1);
	if (var_wn) *var_wn = orc_white_noise_variance(acf, at, ax, ay, phi, pt, px, py);
	return 0;
}
