// Nonlinear inertialess transform (NIT) of a Gaussian surface to a target
// distribution: each value z becomes y with F_target(y) = Phi_sigma(z)
// (reference src/nonlinear/transforms.hh:58-75 driven by
// src/nonlinear/nit_transform.cc:147-168).
//
// Two forms:
//   bisection  the reference's per-point bisection (src/linalg.hh:199-213):
//              midpoint, evaluate f(c), move the bracket by the sign of
//              f(a)*f(c) and f(b)*f(c), stop after max_iter iterations or when
//              the bracket is no wider than eps or |f(c)| <= eps.  FP64.
//   LUT        a pointwise map through an FP64-built inverse-CDF table with
//              cubic Lagrange interpolation between nodes and linear
//              extrapolation beyond the end nodes, stored per interval as
//              power-basis coefficients (one vector load and three FMAs per
//              value).  HBM-bound: one read and one write per value.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "distributions.h"
#include "internal.h"

namespace armab {
namespace {

constexpr int kThreads = 256;

__constant__ dist::GL20 c_gl20;

template <class T>
__global__ void __launch_bounds__(kThreads)
nit_bisection_kernel(T* __restrict__ z, unsigned long long n, int d, double p0, double p1,
                     double p2, double stdev, double a0, double b0, double eps,
                     int max_iter) {
	const double p[3] = {p0, p1, p2};
	const dist::GL20& g = c_gl20;
	for (unsigned long long idx = blockIdx.x * (unsigned long long)kThreads + threadIdx.x;
	     idx < n; idx += (unsigned long long)gridDim.x * kThreads) {
		const double target = dist::gaussian_cdf(double(z[idx]), 0.0, stdev);
		double a = a0, b = b0, c, fc;
		int i = 0;
		do {
			c = 0.5 * (a + b);
			fc = dist::target_cdf(d, p, c, g) - target;
			if ((dist::target_cdf(d, p, a, g) - target) * fc < 0.0) b = c;
			if ((dist::target_cdf(d, p, b, g) - target) * fc < 0.0) a = c;
			i++;
		} while (i < max_iter && (b - a) > eps && fabs(fc) > eps);
		z[idx] = T(c);
	}
}

// The table map over n values: groups of kLutPer 16-byte vectors per thread,
// all loaded before any is mapped (the loads in flight together); the ragged
// head and tail before / after the vectors scalar.  The coefficient table is
// staged in shared memory when it fits (smem = true), else read through L1.
template <class T> struct LutVec;
template <> struct LutVec<float> { using type = float4; static constexpr int n = 4; };
template <> struct LutVec<double> { using type = double2; static constexpr int n = 2; };
constexpr int kLutPer = 4;
constexpr size_t kLutSmemMax = 48 * 1024;

template <class T>
__global__ void __launch_bounds__(kThreads)
nit_lut_kernel(T* __restrict__ z, unsigned long long n,
               const typename NitCoef<T>::type* __restrict__ table, int nodes, T x0, T inv_dx,
               int smem) {
	using C = typename NitCoef<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const C* coef = table;
	if (smem) {
		C* s = reinterpret_cast<C*>(smem_raw);
		for (int i = threadIdx.x; i <= nodes; i += kThreads) s[i] = table[i];
		__syncthreads();
		coef = s;
	}
	using V = typename LutVec<T>::type;
	constexpr int W = LutVec<T>::n;
	// head: values before the first 16-byte boundary
	const unsigned long long head =
	    min(n, (unsigned long long)((16 - (reinterpret_cast<uintptr_t>(z) & 15)) & 15) / sizeof(T));
	const unsigned long long gtid = blockIdx.x * (unsigned long long)kThreads + threadIdx.x;
	const unsigned long long nthr = (unsigned long long)gridDim.x * kThreads;
	if (gtid < head) z[gtid] = nit_lut_map(z[gtid], coef, nodes, x0, inv_dx);
	V* zv = reinterpret_cast<V*>(z + head);
	const unsigned long long nv = (n - head) / W;
	for (unsigned long long base = gtid; base < nv; base += nthr * kLutPer) {
		V v[kLutPer];
#pragma unroll
		for (int r = 0; r < kLutPer; ++r) {
			const unsigned long long i = base + r * nthr;
			if (i < nv) v[r] = zv[i];
		}
#pragma unroll
		for (int r = 0; r < kLutPer; ++r) {
			const unsigned long long i = base + r * nthr;
			if (i < nv) {
				T* e = reinterpret_cast<T*>(&v[r]);
#pragma unroll
				for (int k = 0; k < W; ++k) e[k] = nit_lut_map(e[k], coef, nodes, x0, inv_dx);
				zv[i] = v[r];
			}
		}
	}
	for (unsigned long long i = head + nv * W + gtid; i < n; i += nthr)
		z[i] = nit_lut_map(z[i], coef, nodes, x0, inv_dx);
}

void upload_gl20(Ctx* c) {
	static bool done[64] = {false};
	if (c->device >= 0 && c->device < 64 && !done[c->device]) {
		const dist::GL20& g = dist::gl20_host();
		ARMA_CUDA_TRY(cudaMemcpyToSymbol(c_gl20, &g, sizeof(g)));
		done[c->device] = true;
	}
}

int grid_for(unsigned long long n, int sms) {
	const unsigned long long b = (n + kThreads - 1) / kThreads;
	return int(b < (unsigned long long)(sms * 8) ? (b ? b : 1) : sms * 8);
}

}  // namespace

void launch_nit_bisection(Ctx* c, int d, const double params[3], double stdev, double a,
                          double b, double eps, int max_iter, uint64_t n, int precision,
                          void* d_zeta) {
	ProfScope prof_(c, "nit");
	upload_gl20(c);
	// An iteration either moves one end of the bracket to a midpoint strictly
	// inside it, or leaves the bracket, and so every later iteration, as it
	// is.  A bracket of finite doubles can be halved at most ~2100 times
	// (2^1024 down to the subnormal spacing 2^-1074) before its midpoint
	// rounds to an end, so iterations past 4096 never change the result:
	// larger counts are cut there, which bounds the kernel's run time without
	// changing any output.
	const int iters = std::min(max_iter, 4096);
	const int grid = grid_for(n, c->num_sms);
	if (precision == ARMA_FP64)
		nit_bisection_kernel<double><<<grid, kThreads, 0, c->stream>>>(
		    static_cast<double*>(d_zeta), n, d, params[0], params[1], params[2], stdev, a, b,
		    eps, iters);
	else
		nit_bisection_kernel<float><<<grid, kThreads, 0, c->stream>>>(
		    static_cast<float*>(d_zeta), n, d, params[0], params[1], params[2], stdev, a, b,
		    eps, iters);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

void launch_nit_lut(Ctx* c, const void* d_coef, int nodes, double x0, double dx,
                    uint64_t n, int precision, void* d_zeta) {
	ProfScope prof_(c, "nit");
	ARMA_REQUIRE(nodes >= 4, ARMA_EINVAL, "NIT table needs at least 4 nodes");
	const int grid = grid_for(n, c->num_sms);
	if (precision == ARMA_FP64) {
		const size_t bytes = sizeof(double4) * (size_t(nodes) + 1);
		const bool smem = bytes <= kLutSmemMax;
		nit_lut_kernel<double><<<grid, kThreads, smem ? bytes : 0, c->stream>>>(
		    static_cast<double*>(d_zeta), n, static_cast<const double4*>(d_coef), nodes, x0,
		    1.0 / dx, smem);
	} else {
		const size_t bytes = sizeof(float4) * (size_t(nodes) + 1);
		const bool smem = bytes <= kLutSmemMax;
		nit_lut_kernel<float><<<grid, kThreads, smem ? bytes : 0, c->stream>>>(
		    static_cast<float*>(d_zeta), n, static_cast<const float4*>(d_coef), nodes,
		    float(x0), float(1.0 / dx), smem);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

}  // namespace armab
