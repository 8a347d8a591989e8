// Oracle (test infrastructure): the causal 3-D AR filter, the OpenMP block
// wavefront that the reference uses as its parallel CPU backend, and the
// variance renormalisation.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <mutex>
#include <random>
#include <vector>

namespace {

// Reference: src/generator/ar_model_surf.cc:5-36.  In place over a
// sub-domain [lo, hi] (inclusive); boundary truncation m_d = min(idx+1, p_d);
// k, i, j loop order with a running sum that includes the phi(0,0,0) = 0
// term; zeta += sum.
template <class T>
void ar_box(T* zeta, int nx, int ny, const T* phi, int pt, int px, int py,
            const int lo[3], const int hi[3]) {
	const size_t sx = size_t(ny), st = size_t(nx) * ny;
	for (int t = lo[0]; t <= hi[0]; ++t) {
		for (int x = lo[1]; x <= hi[1]; ++x) {
			for (int y = lo[2]; y <= hi[2]; ++y) {
				const int m1 = std::min(t + 1, pt);
				const int m2 = std::min(x + 1, px);
				const int m3 = std::min(y + 1, py);
				T sum = 0;
				for (int k = 0; k < m1; ++k)
					for (int i = 0; i < m2; ++i)
						for (int j = 0; j < m3; ++j)
							sum += phi[(size_t(k) * px + i) * py + j] *
							       zeta[size_t(t - k) * st + size_t(x - i) * sx + size_t(y - j)];
				zeta[size_t(t) * st + size_t(x) * sx + y] += sum;
			}
		}
	}
}

// Mersenne Twister engine over a dcmt parameter set (same recurrence as
// mt_noise.cc; duplicated here to keep the wavefront self-contained).
struct Engine {
	using result_type = uint32_t;
	orc_mt_params p;
	std::vector<uint32_t> st;
	int i = 0;
	static constexpr result_type min() { return 0; }
	static constexpr result_type max() { return 0xffffffffu; }
	void seed(uint32_t s) {
		st.assign(p.nn, 0);
		for (int k = 0; k < p.nn; ++k) {
			st[k] = s;
			s = 1812433253u * (s ^ (s >> 30)) + uint32_t(k + 1);
		}
		i = p.nn;
		for (int k = 0; k < p.nn; ++k) st[k] &= p.wmask;
	}
	result_type operator()() {
		const int n = p.nn, m = p.mm;
		if (i >= n) {
			int k = 0;
			for (; k < n - m; ++k) {
				const uint32_t x = (st[k] & p.umask) | (st[k + 1] & p.lmask);
				st[k] = st[k + m] ^ (x >> 1) ^ ((x & 1u) ? p.aaa : 0u);
			}
			for (; k < n - 1; ++k) {
				const uint32_t x = (st[k] & p.umask) | (st[k + 1] & p.lmask);
				st[k] = st[k + m - n] ^ (x >> 1) ^ ((x & 1u) ? p.aaa : 0u);
			}
			const uint32_t x = (st[n - 1] & p.umask) | (st[0] & p.lmask);
			st[n - 1] = st[m - 1] ^ (x >> 1) ^ ((x & 1u) ? p.aaa : 0u);
			i = 0;
		}
		uint32_t y = st[i++];
		y ^= y >> p.shift0;
		y ^= (y << p.shiftB) & p.maskB;
		y ^= (y << p.shiftC) & p.maskC;
		y ^= y >> p.shift1;
		return y;
	}
};

int div_ceil(int a, int b) { return a / b + (a % b == 0 ? 0 : 1); }

}  // namespace

extern "C" void orc_ar_filter(double* zeta, int nt, int nx, int ny,
                              const double* phi, int pt, int px, int py) {
	const int lo[3] = {0, 0, 0}, hi[3] = {nt - 1, nx - 1, ny - 1};
	ar_box<double>(zeta, nx, ny, phi, pt, px, py, lo, hi);
}

extern "C" void orc_ar_filter_f32(float* zeta, int nt, int nx, int ny,
                                  const float* phi, int pt, int px, int py) {
	const int lo[3] = {0, 0, 0}, hi[3] = {nt - 1, nx - 1, ny - 1};
	ar_box<float>(zeta, nx, ny, phi, pt, px, py, lo, hi);
}

// Reference: src/generator/ar_model.cc:23-50 (get_partition_shape).
extern "C" void orc_partition_shape(const int grid[3], const int order[3],
                                    int parallelism, const int user[3],
                                    int out[3]) {
	if (user && long(user[0]) * user[1] * user[2] > 0) {
		for (int d = 0; d < 3; ++d) out[d] = user[d];
		return;
	}
	const int npar = std::max(1, 7 * int(std::cbrt(double(parallelism))));
	for (int d = 0; d < 3; ++d) {
		const int g1 = std::max(order[d] * 2, 10);
		const int g2 = div_ceil(grid[d], npar);
		out[d] = std::min(g1, g2) + std::abs(g1 - g2) / 2;
	}
}

// Reference: src/generator/ar_model_parallel.cc:76-201.  Partitions of the
// (t,x,y) box are queued; a thread takes a partition whose [ijk-1, ijk]
// neighbourhood is complete (one mutex + condition variable), fills it with
// white noise from its own MT and a fresh normal_distribution
// (src/generator/ar_model_wn.cc:3-18) when with_noise is set, filters it,
// and marks it complete.
extern "C" int orc_ar_generate_omp(double* zeta, int nt, int nx, int ny,
                                   const double* phi, int pt, int px, int py,
                                   int with_noise, const orc_mt_params* params,
                                   int nparams, const uint32_t* seeds,
                                   double stddev, int nthreads,
                                   const int partition[3]) {
	if (nthreads <= 0) nthreads = omp_get_max_threads();
	if (with_noise && nparams < nthreads) return -1;  // PRNG_error semantics
	const int grid[3] = {nt, nx, ny}, order[3] = {pt, px, py};
	int ps[3];
	orc_partition_shape(grid, order, nthreads, partition, ps);
	int np[3];
	for (int d = 0; d < 3; ++d) np[d] = div_ceil(grid[d], ps[d]);
	struct Part { int ijk[3]; int lo[3]; int hi[3]; };
	std::vector<Part> parts;
	for (int i = 0; i < np[0]; ++i)
		for (int j = 0; j < np[1]; ++j)
			for (int k = 0; k < np[2]; ++k) {
				Part p{{i, j, k}, {}, {}};
				for (int d = 0; d < 3; ++d) {
					p.lo[d] = std::min(p.ijk[d] * ps[d], grid[d]);
					p.hi[d] = std::min((p.ijk[d] + 1) * ps[d], grid[d]) - 1;
				}
				parts.push_back(p);
			}
	std::vector<char> done(size_t(np[0]) * np[1] * np[2], 0);
	auto idx = [&](int i, int j, int k) { return (size_t(i) * np[1] + j) * np[2] + k; };
	std::mutex mtx;
	std::condition_variable cv;
	std::vector<Engine> engines;
	if (with_noise) {
		engines.resize(nthreads);
		for (int t = 0; t < nthreads; ++t) {
			engines[t].p = params[t];
			engines[t].seed(seeds ? seeds[t] : 0u);
		}
	}
	const size_t sx = size_t(ny), st = size_t(nx) * ny;
#pragma omp parallel num_threads(nthreads)
	{
		const int tid = omp_get_thread_num();
		std::unique_lock<std::mutex> lock(mtx);
		while (!parts.empty()) {
			std::vector<Part>::iterator it;
			cv.wait(lock, [&] {
				it = std::find_if(parts.begin(), parts.end(), [&](const Part& p) {
					for (int i = std::max(0, p.ijk[0] - 1); i <= p.ijk[0]; ++i)
						for (int j = std::max(0, p.ijk[1] - 1); j <= p.ijk[1]; ++j)
							for (int k = std::max(0, p.ijk[2] - 1); k <= p.ijk[2]; ++k) {
								if (i == p.ijk[0] && j == p.ijk[1] && k == p.ijk[2]) continue;
								if (!done[idx(i, j, k)]) return false;
							}
					return true;
				});
				return it != parts.end() || parts.empty();
			});
			if (parts.empty()) break;
			Part part = *it;
			parts.erase(it);
			lock.unlock();
			if (with_noise) {
				std::normal_distribution<double> normal(0.0, stddev);
				for (int t = part.lo[0]; t <= part.hi[0]; ++t)
					for (int x = part.lo[1]; x <= part.hi[1]; ++x)
						for (int y = part.lo[2]; y <= part.hi[2]; ++y)
							zeta[size_t(t) * st + size_t(x) * sx + y] = normal(engines[tid]);
			}
			ar_box<double>(zeta, nx, ny, phi, pt, px, py, part.lo, part.hi);
			lock.lock();
			done[idx(part.ijk[0], part.ijk[1], part.ijk[2])] = 1;
			cv.notify_all();
		}
	}
	return 0;
}

// GSL gsl_stats_variance: running mean and running variance in long double
// (x86-64 extended precision), times n/(n-1).
extern "C" double orc_variance_unbiased(const double* x, size_t n) {
	long double mean = 0;
	for (size_t i = 0; i < n; ++i) mean += (x[i] - mean) / (i + 1);
	const double m = double(mean);
	long double var = 0;
	for (size_t i = 0; i < n; ++i) {
		const long double d = (x[i] - m);
		var += (d * d - var) / (i + 1);
	}
	return double(var * ((long double)n / (n - 1)));
}

// Reference: src/generator/basic_arma_model.cc:102-106 with
// src/stats/statistics.hh:35-44.  The statistic is taken through
// variance(Array) = gsl_stats_variance(view.data(), 1, view.numElements()):
// the view zeta(shape/2 : shape-1) is read as numElements() CONTIGUOUS values
// starting at its first element, not as the strided octant.
extern "C" double orc_variance_renorm(double* zeta, int nt, int nx, int ny,
                                      double acf0) {
	const size_t off = (size_t(nt / 2) * nx + nx / 2) * ny + ny / 2;
	const size_t cnt = size_t(nt - nt / 2) * (nx - nx / 2) * (ny - ny / 2);
	const double var = orc_variance_unbiased(zeta + off, cnt);
	const double scale = std::sqrt(acf0 / var);
	const size_t n = size_t(nt) * nx * ny;
	for (size_t i = 0; i < n; ++i) zeta[i] *= scale;
	return scale;
}
