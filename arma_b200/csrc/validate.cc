// Stationarity check of an AR model and the polynomial root finder behind it.
//
// Reference: validate_process (src/arma.cc:14-70) flattens phi into the
// coefficients of the 1-D polynomial 1 - phi_1 x - phi_2 x^2 - ... -
// phi_{P-1} x^{P-1} (phi(0,0,0) is replaced by 1), finds its complex roots
// with gsl_poly_complex_solve, and rejects the process when any root lies
// inside or on the unit circle.  gsl_poly_complex_solve computes the
// eigenvalues of the polynomial's companion matrix after balancing, with the
// Francis double-shift QR iteration on the (already upper Hessenberg)
// matrix; this file restates that published method: Parlett-Reinsch
// balancing by powers of two, then the implicit double-shift QR of an upper
// Hessenberg matrix with deflation on negligible subdiagonal elements and
// exceptional shifts after 10 and 20 iterations.  All FP64.
#include <cmath>
#include <complex>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

// Balances the n x n matrix a (row-major) in place: a diagonal similarity by
// powers of two that makes each row and column norm comparable.
void balance(std::vector<double>& a, int n) {
	auto m = [&](int i, int j) -> double& { return a[size_t(i) * n + j]; };
	const double radix = 2.0, sqr = radix * radix;
	bool changed = true;
	while (changed) {
		changed = false;
		for (int i = 0; i < n; ++i) {
			double c = 0.0, r = 0.0;
			for (int j = 0; j < n; ++j) {
				if (j == i) continue;
				c += std::fabs(m(j, i));
				r += std::fabs(m(i, j));
			}
			if (c == 0.0 || r == 0.0) continue;
			const double total = c + r;
			double f = 1.0, g = r / radix;
			while (c < g) {
				f *= radix;
				c *= sqr;
			}
			g = r * radix;
			while (c > g) {
				f /= radix;
				c /= sqr;
			}
			if ((c + r) / f < 0.95 * total) {
				changed = true;
				for (int j = 0; j < n; ++j) m(i, j) /= f;
				for (int j = 0; j < n; ++j) m(j, i) *= f;
			}
		}
	}
}

// Eigenvalues of the upper Hessenberg n x n matrix h (destroyed).  Returns
// false when an eigenvalue needs more than 60 iterations.
bool hessenberg_eigenvalues(std::vector<double>& h, int n, std::vector<std::complex<double>>& ev) {
	auto a = [&](int i, int j) -> double& { return h[size_t(i) * n + j]; };
	ev.assign(n, 0.0);
	double norm = 0.0;
	for (int i = 0; i < n; ++i)
		for (int j = std::max(i - 1, 0); j < n; ++j) norm += std::fabs(a(i, j));
	int hi = n - 1;
	double shift = 0.0;  // accumulated exceptional shifts
	while (hi >= 0) {
		int its = 0, lo;
		for (;;) {
			// deflation point: the lowest negligible subdiagonal element
			for (lo = hi; lo >= 1; --lo) {
				double s = std::fabs(a(lo - 1, lo - 1)) + std::fabs(a(lo, lo));
				if (s == 0.0) s = norm;
				if (std::fabs(a(lo, lo - 1)) + s == s) {
					a(lo, lo - 1) = 0.0;
					break;
				}
			}
			double x = a(hi, hi);
			if (lo == hi) {  // a 1x1 block
				ev[hi] = x + shift;
				--hi;
				break;
			}
			double y = a(hi - 1, hi - 1);
			double w = a(hi, hi - 1) * a(hi - 1, hi);
			if (lo == hi - 1) {  // a 2x2 block
				const double p = 0.5 * (y - x), q = p * p + w;
				const double z = std::sqrt(std::fabs(q));
				x += shift;
				if (q >= 0.0) {
					const double zz = p + (p >= 0.0 ? z : -z);
					ev[hi - 1] = ev[hi] = x + zz;
					if (zz != 0.0) ev[hi] = x - w / zz;
				} else {
					ev[hi - 1] = std::complex<double>(x + p, z);
					ev[hi] = std::complex<double>(x + p, -z);
				}
				hi -= 2;
				break;
			}
			if (its == 60) return false;
			if (its == 10 || its == 20) {  // exceptional shift
				shift += x;
				for (int i = 0; i <= hi; ++i) a(i, i) -= x;
				const double s = std::fabs(a(hi, hi - 1)) + std::fabs(a(hi - 1, hi - 2));
				x = y = 0.75 * s;
				w = -0.4375 * s * s;
			}
			++its;
			// two consecutive small subdiagonal elements: start of the bulge
			int m;
			double p = 0.0, q = 0.0, r = 0.0;
			for (m = hi - 2; m >= lo; --m) {
				const double z = a(m, m);
				const double rr = x - z, ss = y - z;
				p = (rr * ss - w) / a(m + 1, m) + a(m, m + 1);
				q = a(m + 1, m + 1) - z - rr - ss;
				r = a(m + 2, m + 1);
				const double s = std::fabs(p) + std::fabs(q) + std::fabs(r);
				p /= s;
				q /= s;
				r /= s;
				if (m == lo) break;
				const double u = std::fabs(a(m, m - 1)) * (std::fabs(q) + std::fabs(r));
				const double v =
				    std::fabs(p) * (std::fabs(a(m - 1, m - 1)) + std::fabs(z) + std::fabs(a(m + 1, m + 1)));
				if (u + v == v) break;
			}
			for (int i = m + 2; i <= hi; ++i) {
				a(i, i - 2) = 0.0;
				if (i != m + 2) a(i, i - 3) = 0.0;
			}
			// the implicit double-shift step: chase the bulge down
			for (int k = m; k <= hi - 1; ++k) {
				if (k != m) {
					p = a(k, k - 1);
					q = a(k + 1, k - 1);
					r = k != hi - 1 ? a(k + 2, k - 1) : 0.0;
					x = std::fabs(p) + std::fabs(q) + std::fabs(r);
					if (x != 0.0) {
						p /= x;
						q /= x;
						r /= x;
					}
				}
				const double nrm = std::sqrt(p * p + q * q + r * r);
				const double s = p >= 0.0 ? nrm : -nrm;
				if (s == 0.0) continue;
				if (k == m) {
					if (lo != m) a(k, k - 1) = -a(k, k - 1);
				} else {
					a(k, k - 1) = -s * x;
				}
				p += s;
				x = p / s;
				y = q / s;
				const double z = r / s;
				q /= p;
				r /= p;
				for (int j = k; j <= hi; ++j) {  // rows k..k+2
					double t = a(k, j) + q * a(k + 1, j);
					if (k != hi - 1) {
						t += r * a(k + 2, j);
						a(k + 2, j) -= t * z;
					}
					a(k + 1, j) -= t * y;
					a(k, j) -= t * x;
				}
				const int imax = std::min(hi, k + 3);
				for (int i = lo; i <= imax; ++i) {  // columns k..k+2
					double t = x * a(i, k) + y * a(i, k + 1);
					if (k != hi - 1) {
						t += z * a(i, k + 2);
						a(i, k + 2) -= t * r;
					}
					a(i, k + 1) -= t * q;
					a(i, k) -= t;
				}
			}
		}
	}
	return true;
}

}  // namespace

int poly_roots(const double* c, int n, std::vector<std::complex<double>>& roots) {
	if (n < 2) return 1;
	if (c[n - 1] == 0.0) return 1;  // "leading term of polynomial must be non-zero"
	const int d = n - 1;
	// companion matrix of the monic polynomial: first row -c[d-1-j]/c[d],
	// ones on the subdiagonal
	std::vector<double> m(size_t(d) * d, 0.0);
	for (int j = 0; j < d; ++j) m[j] = -c[d - 1 - j] / c[d];
	for (int i = 1; i < d; ++i) m[size_t(i) * d + i - 1] = 1.0;
	balance(m, d);
	return hessenberg_eigenvalues(m, d, roots) ? 0 : 2;
}

int validate_ar_process(const double* phi, int P, int* bad_roots) {
	*bad_roots = 0;
	if (P <= 1) return 0;
	std::vector<double> c(P);
	c[0] = 1.0;
	for (int k = 1; k < P; ++k) c[k] = -phi[k];
	std::vector<std::complex<double>> roots;
	const int rc = poly_roots(c.data(), P, roots);
	if (rc != 0) return rc;
	for (const auto& z : roots)
		if (!(std::abs(z) > 1.0)) ++*bad_roots;
	return *bad_roots > 0 ? 3 : 0;
}

}  // namespace armab
