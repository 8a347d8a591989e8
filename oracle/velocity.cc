// Oracle (test infrastructure): the linear velocity-potential solver.
#include "oracle.h"

#include <omp.h>

#include <cmath>
#include <complex>
#include <limits>
#include <utility>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double k2Pi = 2.0 * kPi;
constexpr double kG = 9.82;  // src/physical_constants.hh:27

using cplx = std::complex<double>;

// Unnormalised complex DFT along one strided line: sign -1 = forward
// (gsl_fft_forward), +1 = backward (gsl_fft_backward).  Radix-2 for powers of
// two, direct summation otherwise.
void dft_line(cplx* data, int n, int stride, int sign, std::vector<cplx>& buf) {
	buf.resize(n);
	for (int i = 0; i < n; ++i) buf[i] = data[size_t(i) * stride];
	if (n > 1 && (n & (n - 1)) == 0) {
		for (int i = 1, j = 0; i < n; ++i) {
			int bit = n >> 1;
			for (; j & bit; bit >>= 1) j ^= bit;
			j ^= bit;
			if (i < j) std::swap(buf[i], buf[j]);
		}
		for (int len = 2; len <= n; len <<= 1) {
			const int half = len / 2;
			for (int k = 0; k < half; ++k) {
				const double ang = sign * k2Pi * k / len;
				const cplx w(std::cos(ang), std::sin(ang));
				for (int s = 0; s < n; s += len) {
					const cplx u = buf[s + k], v = buf[s + k + half] * w;
					buf[s + k] = u + v;
					buf[s + k + half] = u - v;
				}
			}
		}
		for (int i = 0; i < n; ++i) data[size_t(i) * stride] = buf[i];
	} else {
		for (int k = 0; k < n; ++k) {
			cplx acc(0, 0);
			for (int j = 0; j < n; ++j) {
				const long long m = (long long)j * k % n;
				const double ang = sign * k2Pi * double(m) / n;
				acc += buf[j] * cplx(std::cos(ang), std::sin(ang));
			}
			data[size_t(k) * stride] = acc;
		}
	}
}

// 2-D transform over a C-order (nx, ny) array: columns (dim 0) then rows
// (dim 1), as Fourier_transform::transform does
// (src/apmath/fourier_gsl.hh:140-184).
void fft2(cplx* a, int nx, int ny, int sign) {
	std::vector<cplx> buf;
	for (int j = 0; j < ny; ++j) dft_line(a + j, nx, ny, sign, buf);
	for (int i = 0; i < nx; ++i) dft_line(a + size_t(i) * ny, ny, 1, sign, buf);
}

// Reference: src/interpolate.cc:3-29 (plane through three grid points) and
// src/interpolate.hh:19-35 (evaluate at x).
double interp(const double* f, int ny, int x1a, int x1b, int x2a, int x2b,
              int x3a, int x3b, int xa, int xb) {
	const double f1 = f[size_t(x1a) * ny + x1b];
	const double f2 = f[size_t(x2a) * ny + x2b];
	const double f3 = f[size_t(x3a) * ny + x3b];
	const double c0 =
	    (f2 * x1b - f3 * x1b - f1 * x2b + f3 * x2b + f1 * x3b - f2 * x3b) /
	    (x2a * x1b - x3a * x1b - x1a * x2b + x3a * x2b + x1a * x3b - x2a * x3b);
	const double c1 =
	    (f3 * (-x1a + x2a) + f2 * (x1a - x3a) + f1 * (-x2a + x3a)) /
	    (x3a * (x1b - x2b) + x1a * (x2b - x3b) + x2a * (-x1b + x3b));
	const double c2 =
	    (f3 * x2a * x1b - f2 * x3a * x1b - f3 * x1a * x2b + f1 * x3a * x2b +
	     f2 * x1a * x3b - f1 * x2a * x3b) /
	    (x2a * x1b - x3a * x1b - x1a * x2b + x3a * x2b + x1a * x3b - x2a * x3b);
	return c0 * xa + c1 * xb + c2;
}

struct Event {
	int x = 0, y = 0;
	double period = 0, elevation = 0;
};

// Reference: src/factor_waves.cc:20-73 (factor_waves_dim).  z is accessed as
// z(a, b) = get(a, b) with extents na (first) and nb (second).
template <class Get>
std::pair<double, double> factor_waves_dim(Get get, int na, int nb, int t, double dt) {
	double min_k = std::numeric_limits<double>::max();
	double max_k = std::numeric_limits<double>::min();
	std::vector<Event> events;
	for (int y = 0; y < nb; y++) {
		for (int x = 1; x < na - 1; x++) {
			const double z0 = get(x, y);
			const double z1 = get(x - 1, y);
			const double z2 = get(x + 1, y);
			const double dw1 = z0 - z1;
			const double dw2 = z0 - z2;
			if (!((dw1 > 0.0) ^ (dw2 > 0.0))) {
				const double a = -0.5 * (dw1 + dw2) / (dt * dt);
				const double b = dw1 / dt - a * dt * (2.0 * t - 1.0);
				const double c = z0 - t * dt * (a * t * dt + b);
				const double Tex = -0.5 * b / a;
				const double Wex = c + Tex * (b + a * Tex);
				events.push_back(Event{x, y, Tex, Wex});
			}
		}
	}
	const size_t N = events.size();
	if (N == 0) return {min_k, max_k};  // the reference reads events[0] unguarded
	Event event1 = events[0];
	Event event2;
	size_t j = 0;
	for (size_t i = 1; i < N; i++) {
		if (!((event1.elevation > 0.0) ^ (events[i].elevation > 0.0))) {
			if (std::fabs(event1.elevation) < std::fabs(events[i].elevation)) event1 = events[i];
		} else {
			if (j > 0) {
				const double w = k2Pi / std::fabs((event1.period - event2.period) * 2.0);
				const double k = w * w / kG;
				if (k < min_k) min_k = k;
				if (k > max_k) max_k = k;
			}
			event2 = event1;
			event1 = events[i];
			j++;
		}
	}
	return {min_k, max_k};
}

// blitz::rotate (src/blitz.hh:53-71): column swaps then row swaps.
void rotate(double* r, int nrows, int ncols) {
	const int mr = nrows / 2, mc = ncols / 2;
	for (int i = 0; i < nrows; ++i)
		for (int j = 0; j < mc; ++j)
			std::swap(r[size_t(i) * ncols + j], r[size_t(i) * ncols + (j + mc) % ncols]);
	for (int i = 0; i < mr; ++i)
		for (int j = 0; j < ncols; ++j)
			std::swap(r[size_t(i) * ncols + j], r[size_t((i + mr) % nrows) * ncols + j]);
}

}  // namespace

// Reference: src/derivative.hh:8-73 with dimension 0 (time).
extern "C" void orc_derivative_t(const double* zeta, int nt, int nx, int ny,
                                 double dt, int idx_t, double* out) {
	const size_t st = size_t(nx) * ny;
	const int max_d = nt - 1;
	if (max_d - 0 < 2) {
		for (size_t i = 0; i < st; ++i) out[i] = zeta[size_t(idx_t) * st + i];
		return;
	}
	for (size_t p = 0; p < st; ++p) {
		const double* f = zeta + p;
		const int d = idx_t;
		double r;
		if (d == 0) {
			r = 0.5 * (-f[size_t(d + 2) * st] + 4.0 * f[size_t(d + 1) * st] - 3.0 * f[size_t(d) * st]) / dt;
		} else if (d == max_d) {
			r = 0.5 * (3.0 * f[size_t(d) * st] - 4.0 * f[size_t(d - 1) * st] + f[size_t(d - 2) * st]) / dt;
		} else {
			r = 0.5 * (f[size_t(d + 1) * st] - f[size_t(d - 1) * st]) / dt;
		}
		out[p] = r;
	}
}

// Reference: src/factor_waves.cc:76-89.
extern "C" void orc_factor_waves(const double* s, int nx, int ny, int t, double dt,
                                 double out_min[2], double out_max[2]) {
	auto px = factor_waves_dim([&](int a, int b) { return s[size_t(a) * ny + b]; }, nx, ny, t, dt);
	auto py = factor_waves_dim([&](int a, int b) { return s[size_t(b) * ny + a]; }, ny, nx, t, dt);
	out_min[0] = px.first;
	out_min[1] = py.first;
	out_max[0] = px.second;
	out_max[1] = py.second;
}

// Reference: src/velocity/linear_solver.cc:123-184.  The wave-number grid is
// Domain(wnmax, (nx, ny)): lower bound 0, step ub/(n-1).
extern "C" void orc_window_function(int nx, int ny, double wx, double wy,
                                    double z, double h, double* r) {
	const double dkx = wx / std::max(nx - 1, 1), dky = wy / std::max(ny - 1, 1);
	for (int i = 0; i < nx; ++i)
		for (int j = 0; j < ny; ++j) {
			const double u = 0.0 + dkx * i, v = 0.0 + dky * j;
			const double l = k2Pi * std::sqrt(u * u + v * v);
			const double explz = std::exp(-l * z);
			const double exp2lh = std::exp(-2.0 * l * h);
			const double num = 1.0 + explz * explz * exp2lh;
			const double den = explz * (1.0 + exp2lh);
			r[size_t(i) * ny + j] = k2Pi * 2.0 * num / den;
		}
	double r00 = 0.0;
	int n = 0;
	if (std::isfinite(r[1 * ny + 1])) { r00 += r[1 * ny + 1]; ++n; }
	r00 /= n;
	r[0] = r00;
	for (int i = 1; i < nx; ++i)
		if (!std::isfinite(r[size_t(i) * ny])) r[size_t(i) * ny] = interp(r, ny, i - 1, 1, i, 1, i - 1, 2, i, 0);
	for (int j = 1; j < ny; ++j)
		if (!std::isfinite(r[j])) r[j] = interp(r, ny, 1, j - 1, 1, j, 2, j - 1, 0, j);
	for (size_t i = 0; i < size_t(nx) * ny; ++i)
		if (!std::isfinite(r[i])) r[i] = 0.0;
	rotate(r, nx, ny);
}

extern "C" void orc_fft2(double* re, double* im, int nx, int ny, int sign) {
	std::vector<cplx> a(size_t(nx) * ny);
	for (size_t i = 0; i < a.size(); ++i) a[i] = cplx(re[i], im[i]);
	fft2(a.data(), nx, ny, sign);
	for (size_t i = 0; i < a.size(); ++i) { re[i] = a[i].real(); im[i] = a[i].imag(); }
}

// d zeta / dx (axis 1) or d zeta / dy (axis 2) of slice it, with the
// reference's one-sided differences at the borders and the slice itself when
// the axis has fewer than three points (src/derivative.hh:8-73).
static void derivative_xy(const double* zeta, int nx, int ny, int it, int axis, double d,
                          double* out) {
	const double* f = zeta + size_t(it) * nx * ny;
	const int n = axis == 1 ? nx : ny;
	for (int i = 0; i < nx; ++i)
		for (int j = 0; j < ny; ++j) {
			const int k = axis == 1 ? i : j;
			auto at = [&](int kk) {
				return axis == 1 ? f[size_t(kk) * ny + j] : f[size_t(i) * ny + kk];
			};
			double r;
			if (n - 1 < 2) r = at(k);
			else if (k == 0) r = 0.5 * (-at(2) + 4.0 * at(1) - 3.0 * at(0)) / d;
			else if (k == n - 1) r = 0.5 * (3.0 * at(k) - 4.0 * at(k - 1) + at(k - 2)) / d;
			else r = 0.5 * (at(k + 1) - at(k - 1)) / d;
			out[size_t(i) * ny + j] = r;
		}
}

// Reference: src/velocity/basic_solver.cc:38-77 and 95-112 with the
// Linear_solver hooks (src/velocity/linear_solver.cc:39-121); mode 1 swaps in
// High_amplitude_solver::precompute (src/velocity/high_amplitude_solver.cc:
// 7-23), whose transformed input is the complex
//     d zeta/dt / (i ((zx + zy) / s - zx - zy) - 1 / s),  s = sqrt(1 + zx^2 + zy^2).
// t_idx holds the integer slice indices that the reference obtains by
// truncating the domain's t coordinates; z holds the depth levels.
extern "C" void orc_velocity_solve(int mode, const double* zeta, int nt, int nx, int ny,
                                   const double delta[3], double depth, const double* zs, int nz,
                                   const int* t_idx, int ntd, double* out, int nthreads) {
	if (nthreads <= 0) nthreads = omp_get_max_threads();
	const size_t N = size_t(nx) * ny;
	std::vector<double> zt(N), zx(N), zy(N);
	std::vector<cplx> zc(N);
	for (int i = 0; i < ntd; ++i) {
		const int it = t_idx[i];
		orc_derivative_t(zeta, nt, nx, ny, delta[0], it, zt.data());
		if (mode == 1) {
			derivative_xy(zeta, nx, ny, it, 1, delta[1], zx.data());
			derivative_xy(zeta, nx, ny, it, 2, delta[2], zy.data());
			for (size_t p = 0; p < N; ++p) {
				const double sq = std::sqrt(1.0 + zx[p] * zx[p] + zy[p] * zy[p]);
				zc[p] = zt[p] / cplx(-1.0 / sq, (zx[p] + zy[p]) / sq - zx[p] - zy[p]);
			}
		} else {
			for (size_t p = 0; p < N; ++p) zc[p] = cplx(-zt[p], 0.0);
		}
		double kmin[2], kmax[2];
		// factor_waves(slice, int(t coordinate), dt)
		const int tcoord = int(delta[0] * it);
		orc_factor_waves(zeta + size_t(it) * N, nx, ny, tcoord, delta[0], kmin, kmax);
		const double wx = 1.0 / kmin[0], wy = 1.0 / kmin[1];
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
		for (int j = 0; j < nz; ++j) {
			std::vector<double> w(N);
			orc_window_function(nx, ny, wx, wy, zs[j], depth, w.data());
			std::vector<cplx> a(zc);
			fft2(a.data(), nx, ny, -1);
			for (size_t p = 0; p < N; ++p) a[p] *= w[p];
			fft2(a.data(), nx, ny, +1);
			double* res = out + (size_t(i) * nz + j) * N;
			for (size_t p = 0; p < N; ++p) res[p] = a[p].real() / double(N);
			res[0] = interp(res, ny, 1, 1, 1, 2, 2, 1, 0, 0);
			for (int k = 1; k < nx; ++k)
				res[size_t(k) * ny] = interp(res, ny, k - 1, 1, k, 1, k - 1, 2, k, 0);
			for (int l = 1; l < ny; ++l)
				res[l] = interp(res, ny, 1, l - 1, 1, l, 2, l - 1, 0, l);
		}
	}
}

extern "C" void orc_velocity_linear(const double* zeta, int nt, int nx, int ny,
                                    const double delta[3], double depth, const double* zs, int nz,
                                    const int* t_idx, int ntd, double* out, int nthreads) {
	orc_velocity_solve(0, zeta, nt, nx, ny, delta, depth, zs, nz, t_idx, ntd, out, nthreads);
}
