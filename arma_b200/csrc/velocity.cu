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
// The work is a list of slices (surface pointer, its length, slice index,
// time step, output pointer), so one set of launches serves any number of
// surfaces of one slice shape:
//   1. factor_waves_kernel one CTA per (slice, axis), streaming: extrema
//                          events of a tile of positions are compacted in
//                          loop order with a block scan, then warp 0 walks
//                          them 32 at a time with ballots and a segmented
//                          first-maximum scan, carrying the open sign run
//                          across tiles; min/max k over consecutive closed
//                          runs give wnmax.  No per-event global memory.
//   2a. FP32, nx*ny <= 16384: velocity_fused_kernel, one CTA per slice:
//                          zeta_t into shared memory, in-place radix-2 FFT2
//                          (decimation in frequency: natural in, bit-reversed
//                          out), the spectrum kept in registers, and per depth
//                          the window product in the bit-reversed domain, the
//                          inverse FFT2 (decimation in time: bit-reversed in,
//                          natural out), Re / N and the edge extrapolation,
//                          stored once.
//   2b. otherwise (FP64, larger slices), in passes of bounded scratch:
//                          deriv_kernel -> batched Stockham FFTs through
//                          global memory (rows, then columns) ->
//                          window_mul_kernel -> inverse FFTs -> finish_kernel.
// The window is always evaluated in FP64 with the reference's edge fixes and
// blitz::rotate permutation.
#include <algorithm>
#include <cfloat>
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

// One slice of the work list.
template <class T>
struct VelSlice {
	const T* zeta;  // the surface (slice 0)
	T* out;         // this slice's output: nz planes of nx*ny
	int nt, d;      // surface length, slice index
	double dt;
};

// ---------------------------------------------------------------- 1. zeta_t
// -d zeta/dt at point p of slice s (src/derivative.hh:8-73): central
// differences inside, second-order one-sided differences at both ends, the
// slice itself when the surface has fewer than three slices.
template <class T>
__device__ __forceinline__ double zeta_t(const VelSlice<T>& s, long long n2, long long p) {
	const T* f = s.zeta + p;
	const int d = s.d, nt = s.nt;
	double r;
	if (nt - 1 < 2) {
		r = double(f[d * n2]);
	} else if (d == 0) {
		r = 0.5 * (-double(f[2 * n2]) + 4.0 * double(f[n2]) - 3.0 * double(f[0])) / s.dt;
	} else if (d == nt - 1) {
		r = 0.5 * (3.0 * double(f[d * n2]) - 4.0 * double(f[(d - 1) * n2]) +
		           double(f[(d - 2) * n2])) / s.dt;
	} else {
		r = 0.5 * (double(f[(d + 1) * n2]) - double(f[(d - 1) * n2])) / s.dt;
	}
	return -r;
}

template <class T>
__global__ void deriv_kernel(const VelSlice<T>* __restrict__ sl, int ns, int nx, int ny,
                             typename C2<T>::type* __restrict__ a) {
	const long long n2 = (long long)nx * ny;
	const long long total = n2 * ns;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
	     q += (long long)gridDim.x * blockDim.x) {
		typename C2<T>::type v;
		v.x = T(zeta_t(sl[q / n2], n2, q % n2));
		v.y = T(0);
		a[q] = v;
	}
}

// ---------------------------------------------------------------- 2. wnmax
constexpr int kFwThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int block_scan_excl(int v, int* total, int* sh) {
	// sh: kFwThreads/32 ints
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = v;
	for (int o = 1; o < 32; o <<= 1) {
		const int t = __shfl_up_sync(kFull, incl, o);
		if (lane >= o) incl += t;
	}
	if (lane == 31) sh[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		int s = lane < kFwThreads / 32 ? sh[lane] : 0;
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(kFull, s, o);
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

// The open sign run carried from one group of events to the next (warp 0).
struct RunState {
	bool open = false;     // a run has started
	int sign = 0;          // elevation > 0 of the open run
	double best_e = 0.0;   // |elevation| of the open run's first maximum
	double best_p = 0.0;   // its period
	double prev_p = 0.0;   // first-maximum period of the run before it
	int index = -1;        // index of the open run
	double mn = DBL_MAX, mx = DBL_MIN;
};

__device__ __forceinline__ void pair_k(double p0, double p1, double& mn, double& mx) {
	const double w = k2Pi / fabs((p1 - p0) * 2.0);
	const double k = w * w / kG;
	if (k < mn) mn = k;
	if (k > mx) mx = k;
}

// Events e[0..g) (g <= 32, in loop order) continue the sequence of runs.
// Runs are maximal same-sign stretches; each run's representative is its
// first event of largest |elevation|; every run that closes with index >= 1
// pairs with the run before it (the last run never closes), exactly as the
// reference walks the events one by one.
__device__ void walk_group(const double* ev_p, const double* ev_e, int g, RunState& st) {
	const int lane = threadIdx.x & 31;
	const bool valid = lane < g;
	const double e = valid ? ev_e[lane] : 0.0;
	const double p = valid ? ev_p[lane] : 0.0;
	const int s = e > 0.0 ? 1 : 0;
	const int sprev = __shfl_up_sync(kFull, s, 1);
	bool b = lane == 0 ? (!st.open || s != st.sign) : (s != sprev);
	b = b && valid;
	const unsigned B = __ballot_sync(kFull, b);
	const unsigned upto = B & (lane == 31 ? kFull : ((2u << lane) - 1u));
	const int start = upto ? 31 - __clz(upto) : 0;  // first lane of this lane's run
	// segmented inclusive scan: first maximum of |elevation| within the run
	double bv = fabs(e), bp = p;
	for (int o = 1; o < 32; o <<= 1) {
		const double ov = __shfl_up_sync(kFull, bv, o);
		const double op = __shfl_up_sync(kFull, bp, o);
		if (lane - o >= start && !(bv > ov)) {
			bv = ov;
			bp = op;
		}
	}
	const bool lead = (B & 1u) != 0;  // lane 0 starts a new run
	if (st.open && !lead && upto == 0 && !(bv > st.best_e)) {
		bv = st.best_e;  // the carried run continues: it came first
		bp = st.best_p;
	}
	const int first_index = lead ? (st.open ? st.index + 1 : 0) : st.index;
	const int run = first_index + __popc(upto & ~1u);
	// the previous run's representative for this lane's run
	const double before = __shfl_sync(kFull, bp, start > 0 ? start - 1 : 0);
	const double prev = start > 0 ? before : (lead ? st.best_p : st.prev_p);
	// runs that close inside the group: the carried one (if a new run starts
	// at lane 0) and every run followed by a boundary
	if (lane == 0 && st.open && lead && st.index >= 1) pair_k(st.prev_p, st.best_p, st.mn, st.mx);
	const bool closes = valid && lane + 1 < g && ((B >> (lane + 1)) & 1u);
	if (closes && run >= 1) pair_k(prev, bp, st.mn, st.mx);
	// the run open after the group
	const int last = g - 1;
	const double nbv = __shfl_sync(kFull, bv, last);
	const double nbp = __shfl_sync(kFull, bp, last);
	const int lstart = __shfl_sync(kFull, start, last);
	const int lsign = __shfl_sync(kFull, s, last);
	const int lrun = __shfl_sync(kFull, run, last);
	const double lbefore = __shfl_sync(kFull, bp, lstart > 0 ? lstart - 1 : 0);
	st.prev_p = lstart > 0 ? lbefore : (lead ? st.best_p : st.prev_p);
	st.open = true;
	st.sign = lsign;
	st.best_e = nbv;
	st.best_p = nbp;
	st.index = lrun;
}

// One CTA per (slice, axis).  axis 0 loops y outer, x inner over z(x,y);
// axis 1 (the reference's transposed call) x outer, y inner.  Writes min_k,
// max_k of the axis.
template <class T>
__global__ void __launch_bounds__(kFwThreads)
factor_waves_kernel(const VelSlice<T>* __restrict__ sl, int nx, int ny, double* __restrict__ kout) {
	__shared__ int sh[kFwThreads / 32];
	__shared__ double s_p[kFwThreads], s_e[kFwThreads];
	__shared__ int s_m;
	const int slice = blockIdx.x >> 1, axis = blockIdx.x & 1;
	const VelSlice<T> S = sl[slice];
	const long long n2 = (long long)nx * ny;
	const T* z = S.zeta + S.d * n2;
	const double dt = S.dt;
	const int t = int(dt * S.d);  // factor_waves(slice, int t, dt): the truncated coordinate
	const int outer = axis == 0 ? ny : nx;
	const int inner = (axis == 0 ? nx : ny) - 2;
	const long long L = inner > 0 ? (long long)outer * inner : 0;
	auto at = [&](int a, int b) -> double {  // a: inner index, b: outer index
		return axis == 0 ? double(z[(long long)a * ny + b]) : double(z[(long long)b * ny + a]);
	};
	RunState st;
	for (long long base = 0; base < L; base += kFwThreads) {
		const long long q = base + threadIdx.x;
		int flag = 0;
		double period = 0.0, elevation = 0.0;
		if (q < L) {
			const int b = int(q / inner), a = int(q % inner) + 1;
			const double z0 = at(a, b), z1 = at(a - 1, b), z2 = at(a + 1, b);
			const double dw1 = z0 - z1, dw2 = z0 - z2;
			if (!((dw1 > 0.0) ^ (dw2 > 0.0))) {
				const double aa = -0.5 * (dw1 + dw2) / (dt * dt);
				const double bb = dw1 / dt - aa * dt * (2.0 * t - 1.0);
				const double cc = z0 - t * dt * (aa * t * dt + bb);
				const double tex = -0.5 * bb / aa;
				period = tex;
				elevation = cc + tex * (bb + aa * tex);
				flag = 1;
			}
		}
		int tot;
		const int off = block_scan_excl(flag, &tot, sh);
		if (flag) {
			s_p[off] = period;
			s_e[off] = elevation;
		}
		if (threadIdx.x == 0) s_m = tot;
		__syncthreads();
		if (threadIdx.x < 32) {
			const int m = s_m;
			for (int g0 = 0; g0 < m; g0 += 32) walk_group(s_p + g0, s_e + g0, min(32, m - g0), st);
		}
		__syncthreads();
	}
	if (threadIdx.x < 32) {
		double mn = st.mn, mx = st.mx;
		for (int o = 16; o > 0; o >>= 1) {
			mn = fmin(mn, __shfl_down_sync(kFull, mn, o));
			mx = fmax(mx, __shfl_down_sync(kFull, mx, o));
		}
		if (threadIdx.x == 0) {
			kout[slice * 4 + axis] = mn;      // min_k for this axis
			kout[slice * 4 + 2 + axis] = mx;  // max_k
		}
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
// Re / N with the reference's edge extrapolation (src/velocity/basic_solver.cc:
// 62-68): column 0 (rows >= 1) from columns 1-2, then row 0 from rows 1-2
// reading the fixed column 0, (0,0) from (1,1),(1,2),(2,1).  f(a, c) reads
// Re / N of element (a, c).
template <class F>
__device__ __forceinline__ double finish_at(int x, int y, int nx, int ny, F f) {
	auto col0 = [&](int a) -> double {
		return ny > 2 ? interp3(a - 1, 1, f(a - 1, 1), a, 1, f(a, 1), a - 1, 2, f(a - 1, 2), a, 0)
		              : f(a, 0);
	};
	auto cur = [&](int a, int c) -> double { return c == 0 ? col0(a) : f(a, c); };
	if (x == 0 && y == 0 && nx > 2 && ny > 2)
		return interp3(1, 1, f(1, 1), 1, 2, f(1, 2), 2, 1, f(2, 1), 0, 0);
	if (y == 0 && x > 0) return col0(x);
	if (x == 0 && y > 0 && nx > 2)
		return interp3(1, y - 1, cur(1, y - 1), 1, y, cur(1, y), 2, y - 1, cur(2, y - 1), 0, y);
	return f(x, y);
}

template <class T>
__global__ void finish_kernel(const typename C2<T>::type* __restrict__ b, int nx, int ny,
                              long long narr, int nz, const VelSlice<T>* __restrict__ sl) {
	const long long n2 = (long long)nx * ny;
	const double inv = 1.0 / double(n2);
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < narr * n2;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long arr = q / n2, p = q % n2;
		const int x = int(p / ny), y = int(p % ny);
		const typename C2<T>::type* s = b + arr * n2;
		auto f = [&](int a, int c) -> double { return double(s[(long long)a * ny + c].x) * inv; };
		sl[arr / nz].out[(arr % nz) * n2 + p] = T(finish_at(x, y, nx, ny, f));
	}
}

// ---------------------------------------------------------------- 2a. fused
constexpr int kFuseThreads = 512;
constexpr int kFuseMax = 16384;  // largest nx*ny of the fused path (128 KB of float2)

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }

// In-place radix-2 FFTs of every row (len ny, stride 1) or every column (len
// nx, stride ny) of the nx x ny array in shared memory.  tw[k] =
// exp(-2 pi i k / n), k < n/2.  Forward: decimation in frequency (natural in,
// bit-reversed out); inverse: decimation in time with conjugate twiddles
// (bit-reversed in, natural out).  Unnormalised both ways.
__device__ void fft_rows_dif(float2* a, int nx, int ny, const float2* tw) {
	const int half = ny / 2;
	for (int h = half; h >= 1; h >>= 1) {
		const int tstep = half / h;
		for (int q = threadIdx.x; q < nx * half; q += blockDim.x) {
			const int r = q / half, m = q % half;
			const int j = m & (h - 1);
			const int i0 = r * ny + ((m - j) << 1) + j;
			const float2 u = a[i0], v = a[i0 + h];
			a[i0] = c_add(u, v);
			a[i0 + h] = c_mul(c_sub(u, v), tw[j * tstep]);
		}
		__syncthreads();
	}
}

__device__ void fft_cols_dif(float2* a, int nx, int ny, const float2* tw) {
	const int half = nx / 2;
	for (int h = half; h >= 1; h >>= 1) {
		const int tstep = half / h;
		for (int q = threadIdx.x; q < half * ny; q += blockDim.x) {
			const int c = q % ny, m = q / ny;
			const int j = m & (h - 1);
			const int i0 = (((m - j) << 1) + j) * ny + c;
			const float2 u = a[i0], v = a[i0 + h * ny];
			a[i0] = c_add(u, v);
			a[i0 + h * ny] = c_mul(c_sub(u, v), tw[j * tstep]);
		}
		__syncthreads();
	}
}

__device__ void fft_rows_dit_inv(float2* a, int nx, int ny, const float2* tw) {
	const int half = ny / 2;
	for (int h = 1; h <= half; h <<= 1) {
		const int tstep = half / h;
		for (int q = threadIdx.x; q < nx * half; q += blockDim.x) {
			const int r = q / half, m = q % half;
			const int j = m & (h - 1);
			const int i0 = r * ny + ((m - j) << 1) + j;
			const float2 u = a[i0];
			const float2 v = c_mul(a[i0 + h], c_conj(tw[j * tstep]));
			a[i0] = c_add(u, v);
			a[i0 + h] = c_sub(u, v);
		}
		__syncthreads();
	}
}

__device__ void fft_cols_dit_inv(float2* a, int nx, int ny, const float2* tw) {
	const int half = nx / 2;
	for (int h = 1; h <= half; h <<= 1) {
		const int tstep = half / h;
		for (int q = threadIdx.x; q < half * ny; q += blockDim.x) {
			const int c = q % ny, m = q / ny;
			const int j = m & (h - 1);
			const int i0 = (((m - j) << 1) + j) * ny + c;
			const float2 u = a[i0];
			const float2 v = c_mul(a[i0 + h * ny], c_conj(tw[j * tstep]));
			a[i0] = c_add(u, v);
			a[i0 + h * ny] = c_sub(u, v);
		}
		__syncthreads();
	}
}

__global__ void __launch_bounds__(kFuseThreads, 1)
velocity_fused_kernel(const VelSlice<float>* __restrict__ sl, int nx, int ny, int lnx, int lny,
                      const double* __restrict__ kinfo, const double* __restrict__ zs, int nz,
                      double depth, float2* __restrict__ spectra) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	float2* a = reinterpret_cast<float2*>(smem_raw);  // nx * ny
	float2* twx = a + nx * ny;                         // nx / 2
	float2* twy = twx + nx / 2;                        // ny / 2
	const int s = blockIdx.x;
	const VelSlice<float> S = sl[s];
	const int n2 = nx * ny;
	for (int k = threadIdx.x; k < nx / 2; k += blockDim.x) {
		double sn, cs;
		sincospi(2.0 * k / nx, &sn, &cs);
		twx[k] = make_float2(float(cs), float(-sn));
	}
	for (int k = threadIdx.x; k < ny / 2; k += blockDim.x) {
		double sn, cs;
		sincospi(2.0 * k / ny, &sn, &cs);
		twy[k] = make_float2(float(cs), float(-sn));
	}
	for (int q = threadIdx.x; q < n2; q += blockDim.x)
		a[q] = make_float2(float(zeta_t(S, n2, q)), 0.0f);
	__syncthreads();
	fft_rows_dif(a, nx, ny, twy);
	fft_cols_dif(a, nx, ny, twx);
	// with several depths the spectrum is kept in global memory (L2) and
	// reloaded per depth; the first depth works on it in place
	float2* spec = spectra ? spectra + (long long)s * n2 : nullptr;
	if (spec)
		for (int q = threadIdx.x; q < n2; q += blockDim.x) spec[q] = a[q];
	// wnmax = 1 / min_k per axis; k-grid step ub / (n-1)
	const double wx = 1.0 / kinfo[s * 4 + 0], wy = 1.0 / kinfo[s * 4 + 1];
	const double dkx = wx / max(nx - 1, 1), dky = wy / max(ny - 1, 1);
	const double inv = 1.0 / double(n2);
	for (int iz = 0; iz < nz; ++iz) {
		__syncthreads();  // the previous depth's output read a[]
		for (int q = threadIdx.x; q < n2; q += blockDim.x) {
			// position (i, j) holds frequency (brev i, brev j)
			const int fi = int(__brev(unsigned(q / ny)) >> (32 - lnx));
			const int fj = int(__brev(unsigned(q % ny)) >> (32 - lny));
			const double w = window_fixed(rotate_src(fi, nx), rotate_src(fj, ny), nx, ny, dkx, dky,
			                              zs[iz], depth);
			const float2 x = iz == 0 ? a[q] : spec[q];
			a[q] = make_float2(float(x.x * w), float(x.y * w));
		}
		__syncthreads();
		fft_cols_dit_inv(a, nx, ny, twx);
		fft_rows_dit_inv(a, nx, ny, twy);
		float* out = S.out + (long long)iz * n2;
		auto f = [&](int r, int c) -> double { return double(a[r * ny + c].x) * inv; };
		for (int q = threadIdx.x; q < n2; q += blockDim.x)
			out[q] = float(finish_at(q / ny, q % ny, nx, ny, f));
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

// The general path for one pass of slices: FFTs through global memory.
template <class T>
void velocity_general(Ctx* c, const VelSlice<T>* d_sl, int ns, int nx, int ny, const double* d_k,
                      const double* d_z, int nz, double depth) {
	using V = typename C2<T>::type;
	const long long n2 = (long long)nx * ny;
	V* a = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ns));
	V* b = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ns * nz));
	const int g = c->num_sms * 8;
	deriv_kernel<T><<<g, 256, 0, c->stream>>>(d_sl, ns, nx, ny, a);
	c->launches += 1;
	fft2<T>(c, a, ns, nx, ny, -1);
	window_mul_kernel<T><<<g, 256, 0, c->stream>>>(a, nx, ny, ns, d_k, d_z, nz, depth, b);
	c->launches += 1;
	fft2<T>(c, b, (long long)ns * nz, nx, ny, +1);
	finish_kernel<T><<<g, 256, 0, c->stream>>>(b, nx, ny, (long long)ns * nz, nz, d_sl);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

template <class T>
void velocity_slices(Ctx* c, const std::vector<VelSlice<T>>& slices, int nx, int ny, double depth,
                     const double* z, int nz) {
	ARMA_REQUIRE((nx & (nx - 1)) == 0 && (ny & (ny - 1)) == 0 && nx >= 4 && ny >= 4 &&
	                 nx <= 1024 && ny <= 1024,
	             ARMA_ENOTSUP, "velocity solver: slice sides must be powers of two in [4, 1024]");
	ARMA_REQUIRE(nz >= 1, ARMA_EINVAL, "no z levels");
	const int ns = int(slices.size());
	if (ns == 0) return;
	const long long n2 = (long long)nx * ny;
	auto* d_sl = static_cast<VelSlice<T>*>(scratch_take(c, sizeof(VelSlice<T>) * ns));
	double* d_z = static_cast<double*>(scratch_take(c, sizeof(double) * nz));
	double* d_k = static_cast<double*>(scratch_take(c, sizeof(double) * 4 * ns));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d_sl, slices.data(), sizeof(VelSlice<T>) * ns,
	                              cudaMemcpyHostToDevice, c->stream));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d_z, z, sizeof(double) * nz, cudaMemcpyHostToDevice, c->stream));
	factor_waves_kernel<T><<<2 * ns, kFwThreads, 0, c->stream>>>(d_sl, nx, ny, d_k);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
	if (sizeof(T) == sizeof(float) && n2 <= kFuseMax) {
		const size_t smem = sizeof(float2) * (size_t(n2) + nx / 2 + ny / 2);
		ARMA_CUDA_TRY(cudaFuncSetAttribute(velocity_fused_kernel,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		float2* spectra =
		    nz > 1 ? static_cast<float2*>(scratch_take(c, sizeof(float2) * n2 * ns)) : nullptr;
		velocity_fused_kernel<<<ns, kFuseThreads, smem, c->stream>>>(
		    reinterpret_cast<const VelSlice<float>*>(d_sl), int(nx), int(ny), ilog2(nx), ilog2(ny),
		    d_k, d_z, nz, depth, spectra);
		ARMA_CUDA_TRY(cudaGetLastError());
		c->launches += 1;
		return;
	}
	// passes of at most ~512 MB of complex work buffers
	const long long per_slice = (long long)sizeof(typename C2<T>::type) * n2 * (1 + nz);
	const int pass = int(std::max<long long>(1, std::min<long long>(ns, (512ll << 20) / per_slice)));
	for (int s0 = 0; s0 < ns; s0 += pass) {
		const ScratchMark mark = scratch_mark(c);
		velocity_general<T>(c, d_sl + s0, std::min(pass, ns - s0), nx, ny, d_k + 4 * s0, d_z, nz,
		                    depth);
		scratch_release(c, mark);
	}
}

}  // namespace

void launch_velocity_linear(Ctx* c, const void* d_zeta, const int shape[3], int precision,
                            const double delta[3], double depth, const double* z, int nz,
                            const int* t_idx, int ntd, void* d_out) {
	VelocitySurface v{d_zeta, d_out, shape[0], t_idx, ntd, delta[0]};
	launch_velocity_linear_batch(c, &v, 1, shape[1], shape[2], precision, depth, z, nz);
}

void launch_velocity_linear_batch(Ctx* c, const VelocitySurface* v, int n, int nx, int ny,
                                  int precision, double depth, const double* z, int nz) {
	ProfScope prof_(c, "velocity");
	const long long n2 = (long long)nx * ny;
	if (precision == ARMA_FP64) {
		std::vector<VelSlice<double>> sl;
		for (int k = 0; k < n; ++k)
			for (int i = 0; i < v[k].ntd; ++i)
				sl.push_back(VelSlice<double>{static_cast<const double*>(v[k].zeta),
				                              static_cast<double*>(v[k].out) + (long long)i * nz * n2,
				                              v[k].nt, v[k].t_idx[i], v[k].dt});
		velocity_slices<double>(c, sl, nx, ny, depth, z, nz);
	} else {
		std::vector<VelSlice<float>> sl;
		for (int k = 0; k < n; ++k)
			for (int i = 0; i < v[k].ntd; ++i)
				sl.push_back(VelSlice<float>{static_cast<const float*>(v[k].zeta),
				                             static_cast<float*>(v[k].out) + (long long)i * nz * n2,
				                             v[k].nt, v[k].t_idx[i], v[k].dt});
		velocity_slices<float>(c, sl, nx, ny, depth, z, nz);
	}
}

}  // namespace armab
