// Order-recursive Yule-Walker solver for cubic 3-D AR models (Choi 1999), the
// reference's default fitting algorithm.
//
// Reference: Yule_walker_solver::solve (src/yule_walker.cc:426-539) and
// AR_model::determine_coefficients_choi (src/generator/ar_model.cc:136-152).
// The coefficients are grouped in shells: shell d holds the lags (p,q,r) with
// max(p,q,r) = d, 3d^2+3d+1 of them, in the reference's order (the lag (d,d,d)
// first, then for e = 1..d six runs of e lags each).  Block matrices R(a,b)
// of the normalised ACF between shells a and b (entries rho(|(a-b) - o_a +
// o_b|) per axis, o the shell offsets) drive the recursion: shell by shell
// the solution Pi (one vector per shell), the prediction-error factor lambda
// and the auxiliary matrices Phi(m, a, k) and Theta(m) are updated; the
// recursion stops when the white-noise variance changes by less than
// var_epsilon between orders (or at the maximum order).  Inverses are FP64
// Gauss-Jordan with partial pivoting (the reference uses LAPACK getrf/getri).
#include <cmath>
#include <map>
#include <tuple>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

struct Mat {
	int r = 0, c = 0;
	std::vector<double> a;
	Mat() = default;
	Mat(int rows, int cols) : r(rows), c(cols), a(size_t(rows) * cols, 0.0) {}
	double& operator()(int i, int j) { return a[size_t(i) * c + j]; }
	double operator()(int i, int j) const { return a[size_t(i) * c + j]; }
};

Mat mul(const Mat& x, const Mat& y) {
	Mat z(x.r, y.c);
	for (int i = 0; i < x.r; ++i)
		for (int k = 0; k < x.c; ++k) {
			const double v = x(i, k);
			if (v == 0.0) continue;
			for (int j = 0; j < y.c; ++j) z(i, j) += v * y(k, j);
		}
	return z;
}

std::vector<double> mulv(const Mat& x, const std::vector<double>& v) {
	std::vector<double> z(x.r, 0.0);
	for (int i = 0; i < x.r; ++i) {
		double s = 0.0;
		for (int k = 0; k < x.c; ++k) s += x(i, k) * v[k];
		z[i] = s;
	}
	return z;
}

Mat sub(const Mat& x, const Mat& y) {
	Mat z = x;
	for (size_t i = 0; i < z.a.size(); ++i) z.a[i] -= y.a[i];
	return z;
}

double dot(const std::vector<double>& x, const std::vector<double>& y) {
	double s = 0.0;
	for (size_t i = 0; i < x.size(); ++i) s += x[i] * y[i];
	return s;
}

// In-place inverse (Gauss-Jordan, partial pivoting); false if singular.
bool invert(Mat& m) {
	const int n = m.r;
	Mat inv(n, n);
	for (int i = 0; i < n; ++i) inv(i, i) = 1.0;
	for (int col = 0; col < n; ++col) {
		int piv = col;
		for (int i = col + 1; i < n; ++i)
			if (std::fabs(m(i, col)) > std::fabs(m(piv, col))) piv = i;
		if (m(piv, col) == 0.0) return false;
		if (piv != col)
			for (int j = 0; j < n; ++j) {
				std::swap(m(piv, j), m(col, j));
				std::swap(inv(piv, j), inv(col, j));
			}
		const double d = 1.0 / m(col, col);
		for (int j = 0; j < n; ++j) {
			m(col, j) *= d;
			inv(col, j) *= d;
		}
		for (int i = 0; i < n; ++i) {
			if (i == col) continue;
			const double f = m(i, col);
			if (f == 0.0) continue;
			for (int j = 0; j < n; ++j) {
				m(i, j) -= f * m(col, j);
				inv(i, j) -= f * inv(col, j);
			}
		}
	}
	m = inv;
	return true;
}

struct Off {
	int a, b, c;
};

// Offsets of shell d in the reference's order: the lag of offset o is
// (d,d,d) - o.
std::vector<Off> shell(int d) {
	std::vector<Off> o;
	o.push_back({0, 0, 0});
	for (int e = 1; e <= d; ++e) {
		for (int i = 0; i < e; ++i) o.push_back({e, i, 0});
		for (int i = 0; i < e; ++i) o.push_back({e - i, e, 0});
		for (int i = 0; i < e; ++i) o.push_back({0, e, i});
		for (int i = 0; i < e; ++i) o.push_back({0, e - i, e});
		for (int i = 0; i < e; ++i) o.push_back({i, 0, e});
		for (int i = 0; i < e; ++i) o.push_back({e, 0, e - i});
	}
	return o;
}

class Choi {
public:
	Choi(const double* acf, int n) : n_(n), rho_(acf, acf + size_t(n) * n * n) {
		const double r0 = rho_[0];
		for (double& v : rho_) v /= r0;
	}

	double rho(int i, int j, int k) const {
		i = std::abs(i);
		j = std::abs(j);
		k = std::abs(k);
		return rho_[(size_t(i) * n_ + j) * n_ + k];
	}

	const std::vector<Off>& S(int d) {
		auto it = shells_.find(d);
		if (it == shells_.end()) it = shells_.emplace(d, shell(d)).first;
		return it->second;
	}

	// R(a,b)[n][m] = rho((a-b) - o_a[n] + o_b[m]) per axis; b = 0 gives the
	// column vector of shell a's lags.
	Mat R(int a, int b) {
		const auto& oa = S(a);
		const auto& ob = S(b);
		Mat m(int(oa.size()), int(ob.size()));
		for (size_t p = 0; p < oa.size(); ++p)
			for (size_t q = 0; q < ob.size(); ++q)
				m(int(p), int(q)) = rho(a - b - oa[p].a + ob[q].a, a - b - oa[p].b + ob[q].b,
				                        a - b - oa[p].c + ob[q].c);
		return m;
	}

	std::vector<double> Rcol(int a) { return R(a, 0).a; }  // R(a, 0) as a vector
	std::vector<double> Rrow(int b) { return R(0, b).a; }  // R(0, b) as a vector

private:
	int n_;
	std::vector<double> rho_;
	std::map<int, std::vector<Off>> shells_;
};

// Cube of side `order` from the shell solutions beta[1 .. order-1].
std::vector<double> assemble(const std::vector<std::vector<double>>& beta, int order) {
	std::vector<double> out(size_t(order) * order * order, 0.0);
	for (int d = 1; d < order; ++d) {
		const auto o = shell(d);
		for (size_t n = 0; n < o.size(); ++n) {
			const int i = d - o[n].a, j = d - o[n].b, k = d - o[n].c;
			out[(size_t(i) * order + j) * order + k] = beta[d][n];
		}
	}
	return out;
}

}  // namespace

double ar_white_noise_variance(const double* acf, const int acf_shape[3], const double* phi,
                               const int order[3]) {
	double s = 0.0;
	for (int i = 0; i < order[0]; ++i)
		for (int j = 0; j < order[1]; ++j)
			for (int k = 0; k < order[2]; ++k)
				s += phi[(size_t(i) * order[1] + j) * order[2] + k] *
				     acf[(size_t(i) * acf_shape[1] + j) * acf_shape[2] + k];
	return acf[0] - s;
}

int fit_choi(const double* acf, int n, int max_order, bool determine_order, double var_eps,
             bool chop, double chop_eps, std::vector<double>* phi, int order[3], double* var_out) {
	if (n < 2) return 1;
	max_order = std::min(max_order, n - 1);
	if (max_order < 1) return 1;
	Choi ch(acf, n);
	const double variance = acf[0];
	using Key = std::tuple<int, int, int>;
	std::map<Key, Mat> Phi;
	std::vector<std::vector<double>> Pi_l(max_order + 2), Pi_lp1(max_order + 2);
	std::vector<Mat> Theta(max_order + 2);
	Mat R11inv = ch.R(1, 1);
	if (!invert(R11inv)) return 2;
	Pi_l[1] = mulv(R11inv, ch.Rcol(1));
	double lambda = 1.0 - dot(ch.Rrow(1), Pi_l[1]);
	double var0 = variance, var = variance * lambda;
	Phi[Key(2, 1, 0)] = mul(R11inv, ch.R(1, 2));
	bool changed = false;
	int l = 1;
	do {
		++l;
		var0 = var;
		const int sl = int(ch.S(l).size());
		Mat sum1(sl, sl);
		std::vector<double> sum2(sl, 0.0);
		for (int m = 1; m <= l - 1; ++m) {
			const Mat Rlm = ch.R(l, m);
			const Mat t = mul(Rlm, Phi.at(Key(l, m, 0)));
			for (size_t i = 0; i < t.a.size(); ++i) sum1.a[i] += t.a[i];
			const std::vector<double> u = mulv(Rlm, Pi_l[m]);
			for (size_t i = 0; i < u.size(); ++i) sum2[i] += u[i];
		}
		Mat Th = sub(ch.R(l, l), sum1);
		std::vector<double> h = ch.Rcol(l);
		for (size_t i = 0; i < h.size(); ++i) h[i] -= sum2[i];
		if (!invert(Th)) return 2;
		Theta[l] = Th;
		Pi_lp1[l] = mulv(Th, h);
		for (int a = 1; a <= l - 1; ++a) {
			const std::vector<double> u = mulv(Phi.at(Key(l, a, 0)), Pi_lp1[l]);
			Pi_lp1[a] = Pi_l[a];
			for (size_t i = 0; i < u.size(); ++i) Pi_lp1[a][i] -= u[i];
		}
		lambda -= dot(h, Pi_lp1[l]);
		var = variance * lambda;
		if (l < max_order) {
			Phi[Key(2, 1, l - 1)] = mul(R11inv, ch.R(1, l + 1));
			for (int m = 2; m <= l; ++m) {
				Mat s3 = ch.R(m, l + 1);
				for (int q = 1; q <= m - 1; ++q)
					s3 = sub(s3, mul(ch.R(m, q), Phi.at(Key(m, q, l - m + 1))));
				Phi[Key(m + 1, m, l - m)] = mul(Theta[m], s3);
				for (int a = 1; a <= m - 1; ++a)
					Phi[Key(m + 1, a, l - m)] =
					    sub(Phi.at(Key(m, a, l - m + 1)),
					        mul(Phi.at(Key(m, a, 0)), Phi.at(Key(m + 1, m, l - m))));
			}
		}
		std::swap(Pi_l, Pi_lp1);
		changed = !(determine_order && std::fabs(var - var0) < var_eps);
	} while (l < max_order && changed);
	// the reference keeps the latest solution's shells 1..l-1 when it stopped
	// at the maximum order, else the previous iteration's
	std::vector<double> cube = changed ? assemble(Pi_l, l) : assemble(Pi_lp1, l);
	*var_out = changed ? var : var0;
	int o[3] = {l, l, l};
	if (chop) {  // chop_right (src/chop.cc): drop trailing planes below chop_eps
		auto at = [&](int i, int j, int k) { return std::fabs(cube[(size_t(i) * l + j) * l + k]); };
		auto plane_k = [&](int kk) {
			for (int i = 0; i < l; ++i)
				for (int j = 0; j < l; ++j)
					if (!(at(i, j, kk) < chop_eps)) return false;
			return true;
		};
		int k = l - 1;
		while (k >= 1 && plane_k(k)) --k;
		auto plane_j = [&](int jj) {
			for (int i = 0; i < l; ++i)
				for (int kk = 0; kk <= k; ++kk)
					if (!(at(i, jj, kk) < chop_eps)) return false;
			return true;
		};
		int j = l - 1;
		while (j >= 1 && plane_j(j)) --j;
		auto plane_i = [&](int ii) {
			for (int jj = 0; jj <= j; ++jj)
				for (int kk = 0; kk <= k; ++kk)
					if (!(at(ii, jj, kk) < chop_eps)) return false;
			return true;
		};
		int i = l - 1;
		while (i >= 1 && plane_i(i)) --i;
		o[0] = i + 1;
		o[1] = j + 1;
		o[2] = k + 1;
	}
	phi->assign(size_t(o[0]) * o[1] * o[2], 0.0);
	for (int i = 0; i < o[0]; ++i)
		for (int j = 0; j < o[1]; ++j)
			for (int k = 0; k < o[2]; ++k)
				(*phi)[(size_t(i) * o[1] + j) * o[2] + k] = cube[(size_t(i) * l + j) * l + k];
	for (int q = 0; q < 3; ++q) order[q] = o[q];
	return 0;
}

}  // namespace armab
