// Linear velocity-potential solver on the device.
//
// Reference: Velocity_potential_solver::operator() with the Linear_solver
// hooks (src/velocity/basic_solver.cc:38-112, src/velocity/linear_solver.cc:
// 20-184).  For every requested slice index t and depth z:
//     zeta_t = -d zeta / dt                      (src/derivative.hh:8-73)
//     wnmax  = 1 / min_k from factor_waves       (src/factor_waves.cc:20-89)
//     phi    = Re IFFT2( W(k; wnmax, z, h) . FFT2(zeta_t) ) / (nx ny)
// followed by the 3-point plane extrapolation of row 0 / column 0.
//
// Device decomposition (all slices and depths in a handful of launches):
//   1. deriv_kernel        zeta_t for every slice into a complex buffer A
//   2. factor_waves_kernel one CTA per (slice, axis): extrema events are
//                          compacted in loop order with a block scan, split
//                          into same-sign runs, each run's first maximum of
//                          |elevation| is found, and min/max k over
//                          consecutive run maxima reduce to wnmax
//   3. fft_lines_kernel    batched radix-2 Stockham FFTs in shared memory
//                          (rows, then columns) on A: one forward FFT2 per
//                          slice, shared by all depths
//   4. window_mul_kernel   B[t,z] = A[t] * W_z, the window evaluated per
//                          element with the reference's edge fixes and
//                          blitz::rotate permutation
//   5. fft_lines_kernel    inverse FFT2 of every B[t,z]
//   6. finish_kernel       Re / N and the edge extrapolation into the output
// Complex buffers are float2 for the FP32 form and double2 for FP64.
#include <cmath>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double k2Pi = 2.0 * kPi;
constexpr double kG = 9.82;  // src/physical_constants.hh:27

template <class T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };

template <class V>
__device__ __forceinline__ V cmul(V a, V b) {
	V r;
	r.x = a.x * b.x - a.y * b.y;
	r.y = a.x * b.y + a.y * b.x;
	return r;
}

// ---------------------------------------------------------------- 1. zeta_t
template <class T>
__global__ void deriv_kernel(const T* __restrict__ zeta, int nt, int nx, int ny, double dt,
                             const int* __restrict__ tidx, int ntd,
                             typename C2<T>::type* __restrict__ a) {
	const long long n2 = (long long)nx * ny;
	const long long total = n2 * ntd;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
	     q += (long long)gridDim.x * blockDim.x) {
		const int i = int(q / n2);
		const long long p = q % n2;
		const int d = tidx[i];
		const T* f = zeta + p;
		const long long st = n2;
		double r;
		if (nt - 1 < 2) {
			r = double(f[d * st]);
		} else if (d == 0) {
			r = 0.5 * (-double(f[2 * st]) + 4.0 * double(f[st]) - 3.0 * double(f[0])) / dt;
		} else if (d == nt - 1) {
			r = 0.5 * (3.0 * double(f[d * st]) - 4.0 * double(f[(d - 1) * st]) +
			           double(f[(d - 2) * st])) / dt;
		} else {
			r = 0.5 * (double(f[(d + 1) * st]) - double(f[(d - 1) * st])) / dt;
		}
		typename C2<T>::type v;
		v.x = T(-r);
		v.y = T(0);
		a[q] = v;
	}
}

// ---------------------------------------------------------------- 2. wnmax
struct Event {
	double period, elevation;
};

constexpr int kFwThreads = 512;

__device__ __forceinline__ int block_scan_excl(int v, int* total, int* sh) {
	// sh: kFwThreads/32 ints
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = v;
	for (int o = 1; o < 32; o <<= 1) {
		const int t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += t;
	}
	if (lane == 31) sh[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		int s = lane < kFwThreads / 32 ? sh[lane] : 0;
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += t;
		}
		if (lane < kFwThreads / 32) sh[lane] = s;
	}
	__syncthreads();
	const int base = warp ? sh[warp - 1] : 0;
	*total = sh[kFwThreads / 32 - 1];
	__syncthreads();
	return base + incl - v;
}

// One CTA per (slice, axis).  axis 0: loops y outer, x inner over z(x,y);
// axis 1 (the transposed call): x outer, y inner.  Writes min_k, max_k.
template <class T>
__global__ void __launch_bounds__(kFwThreads)
factor_waves_kernel(const T* __restrict__ zeta, int nx, int ny, const int* __restrict__ tidx,
                    double dt, Event* __restrict__ events_all, int* __restrict__ runs_all,
                    double* __restrict__ kout) {
	__shared__ int sh[kFwThreads / 32];
	__shared__ int s_n, s_runs;
	__shared__ double s_min[kFwThreads / 32], s_max[kFwThreads / 32];
	const int slice = blockIdx.x >> 1, axis = blockIdx.x & 1;
	const int d = tidx[slice];
	const long long n2 = (long long)nx * ny;
	const T* z = zeta + d * n2;
	Event* ev = events_all + (long long)blockIdx.x * n2;
	int* run_start = runs_all + (long long)blockIdx.x * (n2 + 1);
	const int t = int(dt * d);  // factor_waves(slice, int t, dt): t is the truncated coordinate
	const int outer = axis == 0 ? ny : nx;
	const int inner = (axis == 0 ? nx : ny) - 2;
	const long long L = inner > 0 ? (long long)outer * inner : 0;
	auto at = [&](int a, int b) -> double {  // a: inner index, b: outer index
		return axis == 0 ? double(z[(long long)a * ny + b]) : double(z[(long long)b * ny + a]);
	};
	if (threadIdx.x == 0) s_n = 0;
	__syncthreads();
	// compaction of extrema events in loop order
	for (long long base = 0; base < L; base += kFwThreads) {
		const long long q = base + threadIdx.x;
		int flag = 0;
		Event e{0.0, 0.0};
		if (q < L) {
			const int b = int(q / inner), a = int(q % inner) + 1;
			const double z0 = at(a, b), z1 = at(a - 1, b), z2 = at(a + 1, b);
			const double dw1 = z0 - z1, dw2 = z0 - z2;
			if (!((dw1 > 0.0) ^ (dw2 > 0.0))) {
				const double aa = -0.5 * (dw1 + dw2) / (dt * dt);
				const double bb = dw1 / dt - aa * dt * (2.0 * t - 1.0);
				const double cc = z0 - t * dt * (aa * t * dt + bb);
				const double tex = -0.5 * bb / aa;
				const double wex = cc + tex * (bb + aa * tex);
				e.period = tex;
				e.elevation = wex;
				flag = 1;
			}
		}
		int tot;
		const int off = block_scan_excl(flag, &tot, sh);
		if (flag) ev[s_n + off] = e;
		__syncthreads();
		if (threadIdx.x == 0) s_n += tot;
		__syncthreads();
	}
	const int N = s_n;
	// run starts: index 0 and every sign change
	if (threadIdx.x == 0) s_runs = 0;
	__syncthreads();
	for (int base = 0; base < N; base += kFwThreads) {
		const int i = base + threadIdx.x;
		int flag = 0;
		if (i < N) flag = (i == 0) || ((ev[i].elevation > 0.0) != (ev[i - 1].elevation > 0.0));
		int tot;
		const int off = block_scan_excl(flag, &tot, sh);
		if (flag) run_start[s_runs + off] = i;
		__syncthreads();
		if (threadIdx.x == 0) s_runs += tot;
		__syncthreads();
	}
	const int R = s_runs;
	if (threadIdx.x == 0) run_start[R] = N;
	__syncthreads();
	// the first maximum of |elevation| in each run; k between consecutive run
	// maxima r-1, r for r = 1 .. R-2 (the last run is never closed)
	double mn = 1.79769313486231570815e+308, mx = 2.22507385850720138309e-308;
	auto run_max = [&](int r) -> double {
		int best = run_start[r];
		for (int i = best + 1; i < run_start[r + 1]; ++i)
			if (fabs(ev[best].elevation) < fabs(ev[i].elevation)) best = i;
		return ev[best].period;
	};
	for (int r = 1 + threadIdx.x; r <= R - 2; r += kFwThreads) {
		const double p1 = run_max(r), p0 = run_max(r - 1);
		const double w = k2Pi / fabs((p1 - p0) * 2.0);
		const double k = w * w / kG;
		if (k < mn) mn = k;
		if (k > mx) mx = k;
	}
	for (int o = 16; o > 0; o >>= 1) {
		mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
		mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
	}
	if ((threadIdx.x & 31) == 0) {
		s_min[threadIdx.x >> 5] = mn;
		s_max[threadIdx.x >> 5] = mx;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int w = 1; w < kFwThreads / 32; ++w) {
			mn = fmin(mn, s_min[w]);
			mx = fmax(mx, s_max[w]);
		}
		kout[slice * 4 + axis] = mn;      // min_k for this axis
		kout[slice * 4 + 2 + axis] = mx;  // max_k
	}
}

// ---------------------------------------------------------------- 3/5. FFT
// Batched radix-2 Stockham FFT along lines of length n (power of two, <= 1024)
// held in shared memory.  Line l, element k lives at data[line_off(l) +
// k * estride]; a CTA transforms `lines` consecutive line indices whose first
// element is at base + l * lstride within a group of `group` lines, and groups
// are `gstride` apart.
template <class T>
__global__ void fft_lines_kernel(typename C2<T>::type* __restrict__ data, int n, int log2n,
                                 long long nlines, int group, long long lstride,
                                 long long gstride, long long estride, int lines, int sign) {
	using V = typename C2<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	V* buf0 = reinterpret_cast<V*>(smem_raw);
	V* buf1 = buf0 + (size_t)lines * n;
	V* tw = buf1 + (size_t)lines * n;  // n/2 twiddles
	for (int k = threadIdx.x; k < n / 2; k += blockDim.x) {
		double s, c;
		sincospi(2.0 * k / n, &s, &c);
		V w;
		w.x = T(c);
		w.y = T(sign * s);
		tw[k] = w;
	}
	const long long l0 = (long long)blockIdx.x * lines;
	auto addr = [&](long long l, int k) -> long long {
		const long long g = l / group, r = l % group;
		return g * gstride + r * lstride + (long long)k * estride;
	};
	// load: consecutive threads take consecutive lines first when lines are
	// adjacent in memory (column FFTs), else consecutive elements
	const int tot = lines * n;
	for (int q = threadIdx.x; q < tot; q += blockDim.x) {
		int li, k;
		if (lstride == 1) { li = q % lines; k = q / lines; } else { li = q / n; k = q % n; }
		const long long l = l0 + li;
		if (l < nlines) buf0[li * n + k] = data[addr(l, k)];
	}
	__syncthreads();
	V* in = buf0;
	V* out = buf1;
	const int half = n / 2;
	for (int s = 0; s < log2n; ++s) {
		const int Ns = 1 << s;
		for (int q = threadIdx.x; q < lines * half; q += blockDim.x) {
			const int li = q / half, j = q % half;
			const int k = j & (Ns - 1);
			const V a = in[li * n + j];
			V b = in[li * n + j + half];
			b = cmul(b, tw[k * (half / Ns)]);  // exp(sign 2 pi i k / (2 Ns))
			const int o = ((j >> s) << (s + 1)) + k;
			V u, v;
			u.x = a.x + b.x; u.y = a.y + b.y;
			v.x = a.x - b.x; v.y = a.y - b.y;
			out[li * n + o] = u;
			out[li * n + o + Ns] = v;
		}
		__syncthreads();
		V* tmp = in; in = out; out = tmp;
	}
	for (int q = threadIdx.x; q < tot; q += blockDim.x) {
		int li, k;
		if (lstride == 1) { li = q % lines; k = q / lines; } else { li = q / n; k = q % n; }
		const long long l = l0 + li;
		if (l < nlines) data[addr(l, k)] = in[li * n + k];
	}
}

// ---------------------------------------------------------------- 4. window
__device__ __forceinline__ int rotate_src(int i, int n) {
	// blitz::rotate(result, shape/2): swaps j <-> j + n/2 for j < n/2
	const int m = n / 2;
	if (i < m) return i + m;
	if (i < 2 * m) return i - m;
	return i;
}

__device__ double window_raw(int i, int j, double dkx, double dky, double z, double h) {
	const double u = dkx * i, v = dky * j;
	const double l = k2Pi * sqrt(u * u + v * v);
	const double explz = exp(-l * z);
	const double exp2lh = exp(-2.0 * l * h);
	const double num = 1.0 + explz * explz * exp2lh;
	const double den = explz * (1.0 + exp2lh);
	return k2Pi * 2.0 * num / den;
}

// Plane through (x1,f1),(x2,f2),(x3,f3) evaluated at x (src/interpolate.cc:3-29).
__device__ double interp3(int x1a, int x1b, double f1, int x2a, int x2b, double f2, int x3a,
                          int x3b, double f3, int xa, int xb) {
	const double c0 = (f2 * x1b - f3 * x1b - f1 * x2b + f3 * x2b + f1 * x3b - f2 * x3b) /
	                  (x2a * x1b - x3a * x1b - x1a * x2b + x3a * x2b + x1a * x3b - x2a * x3b);
	const double c1 = (f3 * (-x1a + x2a) + f2 * (x1a - x3a) + f1 * (-x2a + x3a)) /
	                  (x3a * (x1b - x2b) + x1a * (x2b - x3b) + x2a * (-x1b + x3b));
	const double c2 = (f3 * x2a * x1b - f2 * x3a * x1b - f3 * x1a * x2b + f1 * x3a * x2b +
	                   f2 * x1a * x3b - f1 * x2a * x3b) /
	                  (x2a * x1b - x3a * x1b - x1a * x2b + x3a * x2b + x1a * x3b - x2a * x3b);
	return c0 * xa + c1 * xb + c2;
}

// Column-0 entry (i >= 1) after the reference's column fix, before zeroing.
__device__ double window_col0(int i, double dkx, double dky, double z, double h) {
	double r = window_raw(i, 0, dkx, dky, z, h);
	if (!isfinite(r))
		r = interp3(i - 1, 1, window_raw(i - 1, 1, dkx, dky, z, h), i, 1,
		            window_raw(i, 1, dkx, dky, z, h), i - 1, 2,
		            window_raw(i - 1, 2, dkx, dky, z, h), i, 0);
	return r;
}

// W(i,j) after the reference's fixes (before rotation): (0,0) from (1,1);
// non-finite column-0 entries from columns 1-2; then non-finite row-0 entries
// from rows 1-2 (which for j = 1 read the already fixed column-0 entries);
// finally every non-finite value becomes 0.
__device__ double window_fixed(int i, int j, int nx, int ny, double dkx, double dky, double z,
                               double h) {
	double r;
	if (i == 0 && j == 0) {
		const double r11 = window_raw(1, 1, dkx, dky, z, h);
		r = isfinite(r11) ? r11 / 1.0 : 0.0 / 0.0;
	} else if (j == 0) {
		r = window_col0(i, dkx, dky, z, h);
	} else {
		r = window_raw(i, j, dkx, dky, z, h);
		if (!isfinite(r) && i == 0) {
			auto cur = [&](int a, int b) {
				return b == 0 ? window_col0(a, dkx, dky, z, h) : window_raw(a, b, dkx, dky, z, h);
			};
			r = interp3(1, j - 1, cur(1, j - 1), 1, j, cur(1, j), 2, j - 1, cur(2, j - 1), 0, j);
		}
	}
	return isfinite(r) ? r : 0.0;
}

template <class T>
__global__ void window_mul_kernel(const typename C2<T>::type* __restrict__ a, int nx, int ny,
                                  int ntd, const double* __restrict__ kinfo,
                                  const double* __restrict__ zs, int nz, double depth,
                                  typename C2<T>::type* __restrict__ b) {
	const long long n2 = (long long)nx * ny;
	const long long total = n2 * ntd * nz;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long p = q % n2;
		const long long iz = q / n2;
		const int j = int(iz % nz), i = int(iz / nz);
		const int x = int(p / ny), y = int(p % ny);
		// wnmax = 1 / min_k per axis; grid step ub / (n-1)
		const double wx = 1.0 / kinfo[i * 4 + 0], wy = 1.0 / kinfo[i * 4 + 1];
		const double dkx = wx / max(nx - 1, 1), dky = wy / max(ny - 1, 1);
		const double w = window_fixed(rotate_src(x, nx), rotate_src(y, ny), nx, ny, dkx, dky,
		                              zs[j], depth);
		typename C2<T>::type v = a[i * n2 + p];
		v.x = T(v.x * w);
		v.y = T(v.y * w);
		b[q] = v;
	}
}

// ---------------------------------------------------------------- 6. finish
template <class T>
__global__ void finish_kernel(const typename C2<T>::type* __restrict__ b, int nx, int ny,
                              long long narr, T* __restrict__ out) {
	const long long n2 = (long long)nx * ny;
	const double inv = 1.0 / double(n2);
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < narr * n2;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long arr = q / n2, p = q % n2;
		const int x = int(p / ny), y = int(p % ny);
		const typename C2<T>::type* s = b + arr * n2;
		auto f = [&](int a, int c) -> double { return double(s[(long long)a * ny + c].x) * inv; };
		// column 0 (rows >= 1) after its fix; row 0 then reads those values
		auto col0 = [&](int a) -> double {
			return ny > 2 ? interp3(a - 1, 1, f(a - 1, 1), a, 1, f(a, 1), a - 1, 2, f(a - 1, 2), a, 0)
			              : f(a, 0);
		};
		auto cur = [&](int a, int c) -> double { return c == 0 ? col0(a) : f(a, c); };
		double r;
		if (x == 0 && y == 0 && nx > 2 && ny > 2) {
			r = interp3(1, 1, f(1, 1), 1, 2, f(1, 2), 2, 1, f(2, 1), 0, 0);
		} else if (y == 0 && x > 0) {
			r = col0(x);
		} else if (x == 0 && y > 0 && nx > 2) {
			r = interp3(1, y - 1, cur(1, y - 1), 1, y, cur(1, y), 2, y - 1, cur(2, y - 1), 0, y);
		} else {
			r = f(x, y);
		}
		out[q] = T(r);
	}
}

int ilog2(int n) {
	int l = 0;
	while ((1 << l) < n) ++l;
	return l;
}

template <class T>
void fft2(Ctx* c, typename C2<T>::type* d, long long narr, int nx, int ny, int sign) {
	using V = typename C2<T>::type;
	const long long n2 = (long long)nx * ny;
	// rows: narr*nx lines of length ny, contiguous
	{
		const int lines = std::max(1, int((48 * 1024 / sizeof(V) - ny / 2) / (2 * ny)));
		const size_t smem = sizeof(V) * (2 * size_t(lines) * ny + ny / 2);
		const long long nlines = narr * nx;
		const int grid = int((nlines + lines - 1) / lines);
		fft_lines_kernel<T><<<grid, 256, smem, c->stream>>>(d, ny, ilog2(ny), nlines, nx, ny, n2, 1,
		                                                      lines, sign);
	}
	// columns: narr*ny lines of length nx, element stride ny
	{
		const int lines = std::max(1, std::min(16, int((48 * 1024 / sizeof(V) - nx / 2) / (2 * nx))));
		const size_t smem = sizeof(V) * (2 * size_t(lines) * nx + nx / 2);
		const long long nlines = narr * ny;
		const int grid = int((nlines + lines - 1) / lines);
		fft_lines_kernel<T><<<grid, 256, smem, c->stream>>>(d, nx, ilog2(nx), nlines, ny, 1, n2, ny,
		                                                      lines, sign);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 2;
}

template <class T>
void velocity_impl(Ctx* c, const T* zeta, const int shape[3], const double delta[3],
                   double depth, const double* z, int nz, const int* t_idx, int ntd, T* out) {
	using V = typename C2<T>::type;
	const int nt = shape[0], nx = shape[1], ny = shape[2];
	ARMA_REQUIRE((nx & (nx - 1)) == 0 && (ny & (ny - 1)) == 0 && nx >= 4 && ny >= 4 &&
	                 nx <= 1024 && ny <= 1024,
	             ARMA_ENOTSUP, "velocity solver: slice sides must be powers of two in [4, 1024]");
	const long long n2 = (long long)nx * ny;
	int* d_tidx = static_cast<int*>(scratch_take(c, sizeof(int) * ntd));
	double* d_z = static_cast<double*>(scratch_take(c, sizeof(double) * nz));
	double* d_k = static_cast<double*>(scratch_take(c, sizeof(double) * 4 * ntd));
	V* a = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ntd));
	V* b = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ntd * nz));
	Event* ev = static_cast<Event*>(scratch_take(c, sizeof(Event) * n2 * 2 * ntd));
	int* runs = static_cast<int*>(scratch_take(c, sizeof(int) * (n2 + 1) * 2 * ntd));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d_tidx, t_idx, sizeof(int) * ntd, cudaMemcpyHostToDevice, c->stream));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d_z, z, sizeof(double) * nz, cudaMemcpyHostToDevice, c->stream));
	const int g = c->num_sms * 8;
	deriv_kernel<T><<<g, 256, 0, c->stream>>>(zeta, nt, nx, ny, delta[0], d_tidx, ntd, a);
	factor_waves_kernel<T><<<2 * ntd, kFwThreads, 0, c->stream>>>(zeta, nx, ny, d_tidx, delta[0],
	                                                              ev, runs, d_k);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 2;
	fft2<T>(c, a, ntd, nx, ny, -1);
	window_mul_kernel<T><<<g, 256, 0, c->stream>>>(a, nx, ny, ntd, d_k, d_z, nz, depth, b);
	c->launches += 1;
	fft2<T>(c, b, (long long)ntd * nz, nx, ny, +1);
	finish_kernel<T><<<g, 256, 0, c->stream>>>(b, nx, ny, (long long)ntd * nz, out);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

}  // namespace

void launch_velocity_linear(Ctx* c, const void* d_zeta, const int shape[3], int precision,
                            const double delta[3], double depth, const double* z, int nz,
                            const int* t_idx, int ntd, void* d_out) {
	ProfScope prof_(c, "velocity");
	if (precision == ARMA_FP64)
		velocity_impl<double>(c, static_cast<const double*>(d_zeta), shape, delta, depth, z, nz,
		                      t_idx, ntd, static_cast<double*>(d_out));
	else
		velocity_impl<float>(c, static_cast<const float*>(d_zeta), shape, delta, depth, z, nz,
		                     t_idx, ntd, static_cast<float*>(d_out));
}

}  // namespace armab
