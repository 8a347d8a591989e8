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
//   1. factor_waves_kernel one CTA per (slice, axis): each lane walks a
//                          piece of one line of the loop order (a column or
//                          a row) and summarises it; the summaries are joined
//                          in a tree.  No per-event global memory.
//   2a. FP32, nx*ny <= 16384: velocity_fused_kernel, one CTA per slice:
//                          zeta_t into shared memory, in-place mixed-radix
//                          FFT2 (decimation in frequency: natural in, digit-
//                          reversed out), and per depth the window product in
//                          the digit-reversed domain, the inverse FFT2
//                          (decimation in time: digit-reversed in, natural
//                          out), Re / N and the edge extrapolation, stored
//                          once.
//   2b. otherwise (FP64, larger slices), in passes of bounded scratch: the
//                          same radix-2 FFTs on bands of rows and columns
//                          held in shared memory, spectra through global
//                          memory between three launches (vel_rows_fwd,
//                          vel_cols with the window, vel_rows_inv).
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


// One slice of the work list.
template <class T>
struct VelSlice {
	const T* zeta;  // the surface (slice 0)
	T* out;         // this slice's output: nz planes of nx*ny
	int nt, d;      // surface length, slice index
	double dt;
	int mode;        // 0 linear, 1 high amplitude
	double dx, dy;   // grid steps for the slope terms of mode 1
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

// d zeta / dx (axis 1) or d zeta / dy (axis 2) at point p of slice s, with
// the same border rules (src/derivative.hh:8-73).
template <class T>
__device__ __forceinline__ double zeta_xy(const VelSlice<T>& s, int nx, int ny, long long p,
                                          int axis) {
	const T* f = s.zeta + (long long)s.d * nx * ny;
	const int i = int(p / ny), j = int(p % ny);
	const int n = axis == 1 ? nx : ny, k = axis == 1 ? i : j;
	const double h = axis == 1 ? s.dx : s.dy;
	auto at = [&](int kk) -> double {
		return axis == 1 ? double(f[(long long)kk * ny + j]) : double(f[(long long)i * ny + kk]);
	};
	if (n - 1 < 2) return at(k);
	if (k == 0) return 0.5 * (-at(2) + 4.0 * at(1) - 3.0 * at(0)) / h;
	if (k == n - 1) return 0.5 * (3.0 * at(k) - 4.0 * at(k - 1) + at(k - 2)) / h;
	return 0.5 * (at(k + 1) - at(k - 1)) / h;
}

// The solver's transformed input at point p: the linear solver's -zeta_t, or
// the high-amplitude solver's d zeta/dt / (i ((zx + zy) / s - zx - zy) - 1/s)
// with s = sqrt(1 + zx^2 + zy^2) (src/velocity/high_amplitude_solver.cc:7-23).
template <class T>
__device__ __forceinline__ void solver_input(const VelSlice<T>& s, int nx, int ny, long long p,
                                             double& re, double& im) {
	const long long n2 = (long long)nx * ny;
	if (s.mode == 0) {
		re = zeta_t(s, n2, p);
		im = 0.0;
		return;
	}
	const double rt = -zeta_t(s, n2, p);
	const double zx = zeta_xy(s, nx, ny, p, 1), zy = zeta_xy(s, nx, ny, p, 2);
	const double sq = sqrt(1.0 + zx * zx + zy * zy);
	const double dr = -1.0 / sq, di = (zx + zy) / sq - zx - zy;
	const double den = dr * dr + di * di;
	re = rt * dr / den;
	im = -rt * di / den;
}

// ---------------------------------------------------------------- 2. wnmax
// factor_waves walks the extrema events of one axis in loop order, splits
// them into maximal same-sign runs, takes each run's first event of largest
// |elevation| as its representative, and forms k = (2 pi / |2 (p_r -
// p_{r-1})|)^2 / g for every run r >= 1 that closes (the last run never
// closes); wnmax comes from the smallest k.
//
// On the device one CTA of kFwThreads threads handles one (slice, axis).  The
// loop order is cut into segments: each line (a column for the x pass, a row
// for the y pass) in P pieces, enough that every warp has work.  A warp walks
// 32 neighbouring lines' pieces at once, one lane per piece, each lane keeping
// the summary of its segment: its runs, the representative periods a join
// still needs and the extreme k of the pairs it closes.  The summaries are then
// joined pairwise in a tree (the join is associative: it is the walk itself
// restarted at a segment boundary) and the pair of the first two runs is added
// at the end.
constexpr int kFwThreads = 256;
constexpr int kFwTile = 35;  // row pitch of the y pass's transposing tile (odd)

struct Run {
	int sign;       // elevation > 0
	double best_e;  // |elevation| of the first maximum
	double best_p;  // its period
};

// Walk state of one segment (uniform over the warp).  Local run indices
// start at 0 with the segment's first run.
struct SegWalk {
	int m = 0;              // runs started so far
	Run open{0, 0.0, 0.0};  // run m-1
	double prev_p = 0.0;    // representative period of run m-2
	Run r0{0, 0.0, 0.0};    // run 0 once closed
	double r1_p = 0.0;      // run 1 once closed
	double mn = DBL_MAX, mx = DBL_MIN;  // pairs (r-1, r) with r >= 2, closed
};

__device__ __forceinline__ void pair_k(double p0, double p1, double& mn, double& mx) {
	const double w = k2Pi / fabs((p1 - p0) * 2.0);
	const double k = w * w / kG;
	if (k < mn) mn = k;
	if (k > mx) mx = k;
}

// One event of a thread's own segment, in loop order.
__device__ __forceinline__ void seg_event(SegWalk& st, double e, double p) {
	const int s = e > 0.0 ? 1 : 0;
	const double ae = fabs(e);
	if (st.m == 0) {
		st.open = Run{s, ae, p};
		st.m = 1;
	} else if (s == st.open.sign) {
		if (st.open.best_e < ae) {  // the first maximum stays
			st.open.best_e = ae;
			st.open.best_p = p;
		}
	} else {
		const int r = st.m - 1;  // the open run closes
		if (r == 0) st.r0 = st.open;
		else if (r == 1) st.r1_p = st.open.best_p;
		else pair_k(st.prev_p, st.open.best_p, st.mn, st.mx);
		st.prev_p = st.open.best_p;
		st.open = Run{s, ae, p};
		++st.m;
	}
}

// The summary of segment A followed by segment B.  B's first run continues
// A's open run when their signs agree (the first maximum stays A's unless B's
// is larger); otherwise A's open run closes at the boundary.  Runs with index
// 0 and 1 keep their representatives for a later join; every other run that
// closes adds its pair.
__device__ SegWalk seg_join(const SegWalk& A, const SegWalk& B) {
	if (A.m == 0) return B;
	if (B.m == 0) return A;
	SegWalk C;
	C.mn = fmin(A.mn, B.mn);
	C.mx = fmax(A.mx, B.mx);
	C.r0 = A.r0;
	C.r1_p = A.r1_p;
	const Run b0 = B.m == 1 ? B.open : B.r0;
	if (b0.sign == A.open.sign) {
		Run R = A.open;  // index A.m - 1
		if (R.best_e < b0.best_e) {
			R.best_e = b0.best_e;
			R.best_p = b0.best_p;
		}
		const int rR = A.m - 1;
		C.m = A.m + B.m - 1;
		if (B.m == 1) {
			C.open = R;
			C.prev_p = A.prev_p;
			return C;
		}
		if (rR == 0) C.r0 = R;
		else if (rR == 1) C.r1_p = R.best_p;
		else pair_k(A.prev_p, R.best_p, C.mn, C.mx);
		if (B.m >= 3) {  // B's run 1 (index rR + 1) closed
			if (rR == 0) C.r1_p = B.r1_p;
			else pair_k(R.best_p, B.r1_p, C.mn, C.mx);
		}
		C.open = B.open;
		C.prev_p = B.m == 2 ? R.best_p : B.prev_p;
		return C;
	}
	const int rA = A.m - 1;  // A's open run closes
	C.m = A.m + B.m;
	if (rA == 0) C.r0 = A.open;
	else if (rA == 1) C.r1_p = A.open.best_p;
	else pair_k(A.prev_p, A.open.best_p, C.mn, C.mx);
	if (B.m == 1) {
		C.open = B.open;
		C.prev_p = A.open.best_p;
		return C;
	}
	if (A.m == 1) C.r1_p = b0.best_p;  // B's run 0 (index A.m) closed
	else pair_k(A.open.best_p, b0.best_p, C.mn, C.mx);
	if (B.m >= 3) pair_k(b0.best_p, B.r1_p, C.mn, C.mx);  // index A.m + 1 >= 2
	C.open = B.open;
	C.prev_p = B.m == 2 ? b0.best_p : B.prev_p;
	return C;
}

// Extremum test and quadratic vertex at position a of a line (z0 = z(a),
// z1 = z(a-1), z2 = z(a+1)), fed to the segment walk.
__device__ __forceinline__ void fw_position(SegWalk& st, double z0, double z1, double z2, double dt,
                                            int t) {
	const double dw1 = z0 - z1, dw2 = z0 - z2;
	if (!((dw1 > 0.0) ^ (dw2 > 0.0))) {
		const double aa = -0.5 * (dw1 + dw2) / (dt * dt);
		const double bb = dw1 / dt - aa * dt * (2.0 * t - 1.0);
		const double cc = z0 - t * dt * (aa * t * dt + bb);
		const double tex = -0.5 * bb / aa;
		seg_event(st, cc + tex * (bb + aa * tex), tex);
	}
}

// Pieces per line: enough (line blocks of 32) x pieces for the CTA's warps,
// at least 8 positions each.
__host__ __device__ inline int fw_pieces(int outer, int npos) {
	const int blocks = (outer + 31) / 32;
	const int want = (kFwThreads / 32 + blocks - 1) / blocks;
	return npos < 16 ? 1 : (want < npos / 8 ? want : npos / 8);
}

// One CTA per (slice, axis).  axis 0 loops y outer, x inner over z(x,y): lane
// b walks column y = b down x (loads coalesced across the warp); axis 1 (the
// reference's transposed call) x outer, y inner: lane b walks row x = b, each
// warp staging 32 rows x 34 columns at a time through shared memory.  Writes
// min_k, max_k of the axis.
template <class T>
__global__ void __launch_bounds__(kFwThreads)
factor_waves_kernel(const VelSlice<T>* __restrict__ sl, int nx, int ny, double* __restrict__ kout) {
	extern __shared__ __align__(16) unsigned char fw_smem[];
	const int slice = blockIdx.x >> 1, axis = blockIdx.x & 1;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
	const VelSlice<T> S = sl[slice];
	const long long n2 = (long long)nx * ny;
	const T* z = S.zeta + S.d * n2;
	const double dt = S.dt;
	const int t = int(dt * S.d);  // factor_waves(slice, int t, dt): the truncated coordinate
	const int outer = axis == 0 ? ny : nx;
	const int npos = (axis == 0 ? nx : ny) - 2;  // positions 1 .. npos of each line
	const int P = fw_pieces(outer, npos), per = (npos + P - 1) / P;
	const int nseg = outer * P, blocks = (outer + 31) / 32;
	SegWalk* seg = reinterpret_cast<SegWalk*>(fw_smem);
	T* tile = reinterpret_cast<T*>(seg + max(nseg, 1)) + warp * 32 * kFwTile;
	for (int u = warp; u < blocks * P; u += nwarps) {
		const int piece = u / blocks, b0 = (u % blocks) * 32, b = b0 + lane;
		const int a_lo = 1 + piece * per, a_hi = 1 + min(npos, (piece + 1) * per);  // [a_lo, a_hi)
		SegWalk st;
		if (axis == 0) {
			if (b < outer && a_lo < a_hi) {
				double z1 = double(z[(long long)(a_lo - 1) * ny + b]);
				double z0 = double(z[(long long)a_lo * ny + b]);
				for (int a = a_lo; a < a_hi; ++a) {
					const double z2 = double(z[(long long)(a + 1) * ny + b]);
					fw_position(st, z0, z1, z2, dt, t);
					z1 = z0;
					z0 = z2;
				}
			}
		} else {
			const int rows = min(32, outer - b0);
			for (int c0 = a_lo; c0 < a_hi; c0 += 32) {
				// columns c0-1 .. c0+32 of rows b0 .. b0+rows-1 (those < ny)
				__syncwarp();
				for (int r = 0; r < rows; ++r) {
					const T* zr = z + (long long)(b0 + r) * ny;
					if (c0 - 1 + lane < ny) tile[r * kFwTile + lane] = zr[c0 - 1 + lane];
					if (lane < 2 && c0 + 31 + lane < ny) tile[r * kFwTile + 32 + lane] = zr[c0 + 31 + lane];
				}
				__syncwarp();
				if (b < outer) {
					const T* row = tile + lane * kFwTile;  // row[k] = z(b, c0 - 1 + k)
					double z1 = double(row[0]), z0 = double(row[1]);
					const int n = min(32, a_hi - c0);
					for (int k = 0; k < n; ++k) {
						const double z2 = double(row[k + 2]);
						fw_position(st, z0, z1, z2, dt, t);
						z1 = z0;
						z0 = z2;
					}
				}
			}
		}
		if (b < outer) seg[b * P + piece] = st;  // loop order: line, then piece
	}
	__syncthreads();
	for (int stride = 1; stride < nseg; stride <<= 1) {
		for (int i = threadIdx.x * 2 * stride; i + stride < nseg; i += blockDim.x * 2 * stride)
			seg[i] = seg_join(seg[i], seg[i + stride]);
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		SegWalk all = nseg > 0 ? seg[0] : SegWalk{};
		if (all.m >= 3) pair_k(all.r0.best_p, all.r1_p, all.mn, all.mx);  // runs 0 and 1
		kout[slice * 4 + axis] = all.mn;      // min_k for this axis
		kout[slice * 4 + 2 + axis] = all.mx;  // max_k
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
	// the exponentials' exact values where the argument is exactly 0 (z = 0)
	// or -inf (infinite depth) skip the FP64 exp; l = 0 at infinite depth
	// still gives exp(NaN) = NaN, as in the reference
	const double az = -l * z, ah = -2.0 * l * h;
	const double explz = az == 0.0 ? 1.0 : exp(az);
	const double exp2lh = ah == -INFINITY ? 0.0 : exp(ah);
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

// ---------------------------------------------------------------- 2a. fused
constexpr int kFuseThreads = 512;
constexpr int kFuseMax = 16384;  // largest nx*ny of the fused path (128 KB of float2)

__device__ __forceinline__ float2 cpx(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 cpx(double x, double y) { return make_double2(x, y); }
template <class V>
__device__ __forceinline__ V c_add(V a, V b) { return cpx(a.x + b.x, a.y + b.y); }
template <class V>
__device__ __forceinline__ V c_sub(V a, V b) { return cpx(a.x - b.x, a.y - b.y); }
template <class V>
__device__ __forceinline__ V c_mul(V a, V b) {
	return cpx(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class V>
__device__ __forceinline__ V c_conj(V a) { return cpx(a.x, -a.y); }

// ---------------------------------------------------------------- FFT
// In-place mixed-radix FFTs of lines held in shared memory (any length <=
// 1024 whose prime factors are <= kMaxRadix; GSL's mixed-radix transform in
// the reference takes any length).  A plan lists the radices of the forward
// stages.  Forward: decimation in frequency -- stage s splits each block of
// L_s points into r_s interleaved sub-blocks of h_s = L_s / r_s, applies the
// r_s-point DFT across them and the twiddles W_{L_s}^{q j}; the output is in
// digit-reversed order (position sum q_s h_s holds frequency sum q_s
// r_0...r_{s-1}).  Inverse: the mirror stages in reverse order (conjugate
// twiddles, then the conjugate r_s-point DFT), digit-reversed in, natural out.
// Unnormalised both ways.  tw[k] = exp(-2 pi i k / n), k < n, from FP64
// sincospi.
constexpr int kMaxStages = 12;
constexpr int kMaxRadix = 64;

struct FftPlan {
	int n, m;
	int r[kMaxStages];
};

template <class V>
__device__ void make_twiddles(V* tw, int n) {
	for (int k = threadIdx.x; k < n; k += blockDim.x) {
		double sn, cs;
		sincospi(2.0 * k / n, &sn, &cs);
		tw[k] = cpx(decltype(tw[0].x)(cs), decltype(tw[0].x)(-sn));
	}
}

// Frequency held at position p after the forward stages.
__device__ __forceinline__ int plan_freq(const FftPlan& P, int p) {
	int h = P.n, w = 1, f = 0;
	for (int s = 0; s < P.m; ++s) {
		h /= P.r[s];
		f += ((p / h) % P.r[s]) * w;
		w *= P.r[s];
	}
	return f;
}

// R-point DFT of v[0..R) in place: forward roots exp(-2 pi i t / R) (= tw[t
// n/R], rs = n/R), conjugated for the inverse.  Fixed R: registers.
template <class V, bool INV, int R>
__device__ __forceinline__ void dft_fixed(V* v, int rs, const V* tw) {
	using T = decltype(v[0].x);
	if constexpr (R == 2) {
		const V a = v[0], b = v[1];
		v[0] = c_add(a, b);
		v[1] = c_sub(a, b);
	} else if constexpr (R == 4) {
		const V t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
		const V t2 = c_add(v[1], v[3]);
		const V d = c_sub(v[1], v[3]);
		const V t3 = INV ? cpx(-d.y, d.x) : cpx(d.y, -d.x);  // (+-i) d
		v[0] = c_add(t0, t2);
		v[1] = c_add(t1, t3);
		v[2] = c_sub(t0, t2);
		v[3] = c_sub(t1, t3);
	} else if constexpr (R == 3) {
		const T c = T(-0.5), sn = INV ? T(0.86602540378443864676) : T(-0.86602540378443864676);
		const V t1 = c_add(v[1], v[2]), t2 = c_sub(v[1], v[2]);
		const V m = cpx(v[0].x + c * t1.x, v[0].y + c * t1.y);
		const V it = cpx(-sn * t2.y, sn * t2.x);  // i sn t2
		v[0] = c_add(v[0], t1);
		v[1] = c_add(m, it);
		v[2] = c_sub(m, it);
	} else {
		V y[R];
#pragma unroll
		for (int q = 0; q < R; ++q) {
			V acc = v[0];
#pragma unroll
			for (int k = 1; k < R; ++k) {
				const V w = tw[((q * k) % R) * rs];
				acc = c_add(acc, c_mul(v[k], INV ? c_conj(w) : w));
			}
			y[q] = acc;
		}
#pragma unroll
		for (int q = 0; q < R; ++q) v[q] = y[q];
	}
}

// One radix-R butterfly of a stage: elements x[k hs], k < R, of sub-block
// offset j; twiddles W_L^{k j} = tw[k j tws].
template <class V, bool INV, int R>
__device__ __forceinline__ void butterfly(V* x, int hs, int j, int tws, int rs, const V* tw) {
	V v[R];
#pragma unroll
	for (int k = 0; k < R; ++k) v[k] = x[k * hs];
	if (INV) {
#pragma unroll
		for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], c_conj(tw[k * j * tws]));
	}
	dft_fixed<V, INV, R>(v, rs, tw);
	if (!INV) {
#pragma unroll
		for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], tw[k * j * tws]);
	}
#pragma unroll
	for (int k = 0; k < R; ++k) x[k * hs] = v[k];
}

// Any other radix (a prime <= kMaxRadix): the DFT by direct summation.
template <class V, bool INV>
__device__ __noinline__ void butterfly_any(V* x, int hs, int r, int j, int tws, int rs,
                                           const V* tw) {
	V v[kMaxRadix], y[kMaxRadix];
	for (int k = 0; k < r; ++k) {
		v[k] = x[k * hs];
		if (INV && k > 0) v[k] = c_mul(v[k], c_conj(tw[k * j * tws]));
	}
	for (int q = 0; q < r; ++q) {
		V acc = v[0];
		for (int k = 1; k < r; ++k) {
			const V w = tw[((q * k) % r) * rs];
			acc = c_add(acc, c_mul(v[k], INV ? c_conj(w) : w));
		}
		y[q] = (!INV && q > 0) ? c_mul(acc, tw[q * j * tws]) : acc;
	}
	for (int q = 0; q < r; ++q) x[q * hs] = y[q];
}

// Every stage over `nlines` lines: line l, element e at a[l * lstride + e *
// estride].  lines_fastest puts consecutive threads on consecutive lines
// (column transforms), else on consecutive elements (row transforms); with
// rows_padded (row transforms whose line stride is an odd number of
// elements) stages of span h < 32 also go lines-first, which keeps their
// butterflies free of shared-memory bank conflicts.
template <class V, bool INV>
__device__ void fft_lines(V* a, int nlines, int lstride, int estride, const FftPlan& P,
                          const V* tw, bool lines_fastest, bool rows_padded = false) {
	const int n = P.n;
	for (int si = 0; si < P.m; ++si) {
		const int s = INV ? P.m - 1 - si : si;
		int L = n;
		for (int t = 0; t < s; ++t) L /= P.r[t];
		const int r = P.r[s], h = L / r, per = (n / L) * h;
		const int tws = n / L, rs = n / r;
		const bool lf = lines_fastest || (rows_padded && h < 32 && nlines >= 8);
		for (int q = threadIdx.x; q < nlines * per; q += blockDim.x) {
			int line, bj;
			if (lf) {
				line = q % nlines;
				bj = q / nlines;
			} else {
				line = q / per;
				bj = q % per;
			}
			const int b = bj / h, j = bj % h;
			V* x = a + line * lstride + (b * L + j) * estride;
			const int hs = h * estride;
			switch (r) {
				case 4: butterfly<V, INV, 4>(x, hs, j, tws, rs, tw); break;
				case 2: butterfly<V, INV, 2>(x, hs, j, tws, rs, tw); break;
				case 3: butterfly<V, INV, 3>(x, hs, j, tws, rs, tw); break;
				case 5: butterfly<V, INV, 5>(x, hs, j, tws, rs, tw); break;
				case 7: butterfly<V, INV, 7>(x, hs, j, tws, rs, tw); break;
				default: butterfly_any<V, INV>(x, hs, r, j, tws, rs, tw); break;
			}
		}
		__syncthreads();
	}
}

// Window row/column indices of the spectrum positions: position p along an
// axis of length n holds frequency plan_freq(p), whose window index is its
// blitz::rotate source.  Built once per CTA into shared memory.
__device__ void make_window_index(int* idx, const FftPlan& P) {
	for (int p = threadIdx.x; p < P.n; p += blockDim.x) idx[p] = rotate_src(plan_freq(P, p), P.n);
}

__global__ void __launch_bounds__(kFuseThreads, 1)
velocity_fused_kernel(const VelSlice<float>* __restrict__ sl, int nx, int ny, FftPlan px,
                      FftPlan py, const double* __restrict__ kinfo, const double* __restrict__ zs,
                      int nz, double depth, float2* __restrict__ spectra) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int ld = ny + 1;                             // padded row stride
	float2* a = reinterpret_cast<float2*>(smem_raw);  // nx rows of ld
	float2* twx = a + nx * ld;                         // nx
	float2* twy = twx + nx;                            // ny
	int* wix = reinterpret_cast<int*>(twy + ny);       // nx window row indices
	int* wiy = wix + nx;                               // ny window column indices
	const int s = blockIdx.x;
	const VelSlice<float> S = sl[s];
	const int n2 = nx * ny;
	make_twiddles(twx, nx);
	make_twiddles(twy, ny);
	make_window_index(wix, px);
	make_window_index(wiy, py);
	for (int q = threadIdx.x; q < n2; q += blockDim.x)
	{
		double re, im;
		solver_input(S, nx, ny, q, re, im);
		a[(q / ny) * ld + q % ny] = make_float2(float(re), float(im));
	}
	__syncthreads();
	fft_lines<float2, false>(a, nx, ld, 1, py, twy, false, true);  // rows
	fft_lines<float2, false>(a, ny, 1, ld, px, twx, true);         // columns
	// with several depths the spectrum is kept in global memory (L2) and
	// reloaded per depth; the first depth works on it in place
	float2* spec = spectra ? spectra + (long long)s * n2 : nullptr;
	if (spec)
		for (int q = threadIdx.x; q < n2; q += blockDim.x) spec[q] = a[(q / ny) * ld + q % ny];
	// wnmax = 1 / min_k per axis; k-grid step ub / (n-1)
	const double wx = 1.0 / kinfo[s * 4 + 0], wy = 1.0 / kinfo[s * 4 + 1];
	const double dkx = wx / max(nx - 1, 1), dky = wy / max(ny - 1, 1);
	const double inv = 1.0 / double(n2);
	for (int iz = 0; iz < nz; ++iz) {
		__syncthreads();  // the previous depth's output read a[]
		for (int q = threadIdx.x; q < n2; q += blockDim.x) {
			const double w = window_fixed(wix[q / ny], wiy[q % ny], nx, ny, dkx, dky, zs[iz], depth);
			const int qa = (q / ny) * ld + q % ny;
			const float2 x = iz == 0 ? a[qa] : spec[q];
			a[qa] = make_float2(float(x.x * w), float(x.y * w));
		}
		__syncthreads();
		fft_lines<float2, true>(a, ny, 1, ld, px, twx, true);
		fft_lines<float2, true>(a, nx, ld, 1, py, twy, false, true);
		float* out = S.out + (long long)iz * n2;
		auto f = [&](int r, int c) -> double { return double(a[r * ld + c].x) * inv; };
		for (int q = threadIdx.x; q < n2; q += blockDim.x)
			out[q] = float(finish_at(q / ny, q % ny, nx, ny, f));
	}
}

// Radices of the forward stages: 4s first, then 2, 3, 5, 7, ... (at most
// kMaxRadix); false when n has a larger prime factor.
bool make_plan(int n, FftPlan* P) {
	P->n = n;
	P->m = 0;
	int rest = n;
	auto push = [&](int r) {
		if (P->m >= kMaxStages) return false;
		P->r[P->m++] = r;
		rest /= r;
		return true;
	};
	while (rest % 4 == 0)
		if (!push(4)) return false;
	while (rest % 2 == 0)
		if (!push(2)) return false;
	for (int f = 3; rest > 1 && f <= kMaxRadix; f += 2)
		while (rest % f == 0)
			if (!push(f)) return false;
	return rest == 1;
}

// ---------------------------------------------------------------- 2b. banded
// Slices larger than the fused kernel's shared memory go through three
// banded passes with the spectra in global memory (A: one per slice, B: one
// per slice and depth), each band sized to ~64 KB of shared memory:
//   vel_rows_fwd   R rows of zeta_t, forward row FFTs        -> A
//   vel_cols       CB columns of A, forward column FFTs, then per depth the
//                  window product and inverse column FFTs     -> B
//   vel_rows_inv   R rows (+ the row above) of B, inverse row FFTs, Re / N
//                  and the edge extrapolation                  -> output
template <class T>
__global__ void __launch_bounds__(256)
vel_rows_fwd(const VelSlice<T>* __restrict__ sl, int nx, int ny, int R, FftPlan py,
             typename C2<T>::type* __restrict__ A) {
	using V = typename C2<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int ld = ny + 1;                  // padded row stride
	V* a = reinterpret_cast<V*>(smem_raw);  // R rows of ld
	V* tw = a + R * ld;                     // ny
	const long long n2 = (long long)nx * ny;
	const VelSlice<T> S = sl[blockIdx.y];
	const int r0 = blockIdx.x * R, rows = min(R, nx - r0);
	make_twiddles(tw, ny);
	for (int q = threadIdx.x; q < rows * ny; q += blockDim.x)
	{
		double re, im;
		solver_input(S, nx, ny, (long long)r0 * ny + q, re, im);
		a[(q / ny) * ld + q % ny] = cpx(T(re), T(im));
	}
	__syncthreads();
	fft_lines<V, false>(a, rows, ld, 1, py, tw, false, true);
	V* dst = A + blockIdx.y * n2 + (long long)r0 * ny;
	for (int q = threadIdx.x; q < rows * ny; q += blockDim.x) dst[q] = a[(q / ny) * ld + q % ny];
}

template <class T>
__global__ void __launch_bounds__(256)
vel_cols(int nx, int ny, FftPlan px, FftPlan py, int CB, const double* __restrict__ kinfo,
         const double* __restrict__ zs, int nz, double depth,
         const typename C2<T>::type* __restrict__ A, typename C2<T>::type* __restrict__ B) {
	using V = typename C2<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	V* spec = reinterpret_cast<V*>(smem_raw);  // nx x cols
	V* work = nz > 1 ? spec + nx * CB : spec;  // one buffer when there is one depth
	V* tw = spec + (nz > 1 ? 2 : 1) * nx * CB;  // nx
	int* wix = reinterpret_cast<int*>(tw + nx);  // nx window row indices
	int* wiy = wix + nx;                         // ny window column indices
	const long long n2 = (long long)nx * ny;
	const int s = blockIdx.y, c0 = blockIdx.x * CB, cols = min(CB, ny - c0);
	make_twiddles(tw, nx);
	make_window_index(wix, px);
	make_window_index(wiy, py);
	const V* src = A + s * n2 + c0;
	for (int q = threadIdx.x; q < nx * cols; q += blockDim.x)
		spec[q] = src[(long long)(q / cols) * ny + q % cols];
	__syncthreads();
	fft_lines<V, false>(spec, cols, 1, cols, px, tw, true);
	const double wx = 1.0 / kinfo[s * 4 + 0], wy = 1.0 / kinfo[s * 4 + 1];
	const double dkx = wx / max(nx - 1, 1), dky = wy / max(ny - 1, 1);
	for (int iz = 0; iz < nz; ++iz) {
		for (int q = threadIdx.x; q < nx * cols; q += blockDim.x) {
			const double w = window_fixed(wix[q / cols], wiy[c0 + q % cols], nx, ny, dkx, dky,
			                              zs[iz], depth);
			const V x = spec[q];
			work[q] = cpx(T(x.x * w), T(x.y * w));
		}
		__syncthreads();
		fft_lines<V, true>(work, cols, 1, cols, px, tw, true);
		V* dst = B + ((long long)s * nz + iz) * n2 + c0;
		for (int q = threadIdx.x; q < nx * cols; q += blockDim.x)
			dst[(long long)(q / cols) * ny + q % cols] = work[q];
		__syncthreads();
	}
}

template <class T>
__global__ void __launch_bounds__(256)
vel_rows_inv(const VelSlice<T>* __restrict__ sl, int nx, int ny, int R, int nz, FftPlan py,
             const typename C2<T>::type* __restrict__ B) {
	using V = typename C2<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int ld = ny + 1;                  // padded row stride
	V* a = reinterpret_cast<V*>(smem_raw);  // R + 1 rows of ld: the row above the band first
	V* tw = a + (R + 1) * ld;               // ny
	const long long n2 = (long long)nx * ny;
	const long long arr = blockIdx.y;  // slice * nz + depth
	const int r0 = blockIdx.x * R, rows = min(R, nx - r0);
	make_twiddles(tw, ny);
	const V* src = B + arr * n2;
	for (int q = threadIdx.x; q < (rows + 1) * ny; q += blockDim.x) {
		const int row = r0 - 1 + q / ny;
		a[(q / ny) * ld + q % ny] = row >= 0 ? src[(long long)row * ny + q % ny] : cpx(T(0), T(0));
	}
	__syncthreads();
	fft_lines<V, true>(a, rows + 1, ld, 1, py, tw, false, true);
	const double inv = 1.0 / double(n2);
	auto f = [&](int x, int y) -> double { return double(a[(x - r0 + 1) * ld + y].x) * inv; };
	T* out = sl[arr / nz].out + (arr % nz) * n2 + (long long)r0 * ny;
	for (int q = threadIdx.x; q < rows * ny; q += blockDim.x)
		out[q] = T(finish_at(r0 + q / ny, q % ny, nx, ny, f));
}

// The banded path for one pass of slices.
template <class T>
void velocity_general(Ctx* c, const VelSlice<T>* d_sl, int ns, int nx, int ny, const FftPlan& px,
                      const FftPlan& py, const double* d_k, const double* d_z, int nz,
                      double depth) {
	using V = typename C2<T>::type;
	const long long n2 = (long long)nx * ny;
	const int budget = int((64 << 10) / sizeof(V));  // elements of one 64 KB band
	const int R = std::min(nx, std::max(4, budget / ny));
	const int CB = std::min(ny, std::max(1, budget / nx));
	V* A = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ns));
	V* B = static_cast<V*>(scratch_take(c, sizeof(V) * n2 * ns * nz));
	const size_t s1 = sizeof(V) * (size_t(R) * (ny + 1) + ny);
	const size_t s2 = sizeof(V) * ((nz > 1 ? 2 : 1) * size_t(nx) * CB + nx) +
	                  sizeof(int) * (size_t(nx) + ny);
	const size_t s3 = sizeof(V) * (size_t(R + 1) * (ny + 1) + ny);
	ARMA_CUDA_TRY(cudaFuncSetAttribute(vel_rows_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                   int(s1)));
	ARMA_CUDA_TRY(cudaFuncSetAttribute(vel_cols<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                   int(s2)));
	ARMA_CUDA_TRY(cudaFuncSetAttribute(vel_rows_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                   int(s3)));
	const int bands = (nx + R - 1) / R, cbands = (ny + CB - 1) / CB;
	vel_rows_fwd<T><<<dim3(bands, ns), 256, s1, c->stream>>>(d_sl, nx, ny, R, py, A);
	vel_cols<T><<<dim3(cbands, ns), 256, s2, c->stream>>>(nx, ny, px, py, CB, d_k, d_z, nz, depth,
	                                                       A, B);
	vel_rows_inv<T><<<dim3(bands, ns * nz), 256, s3, c->stream>>>(d_sl, nx, ny, R, nz, py, B);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 3;
}

template <class T>
void velocity_slices(Ctx* c, const std::vector<VelSlice<T>>& slices, int nx, int ny, double depth,
                     const double* z, int nz) {
	FftPlan px, py;
	ARMA_REQUIRE(nx >= 4 && ny >= 4 && nx <= 1024 && ny <= 1024 && make_plan(nx, &px) &&
	                 make_plan(ny, &py),
	             ARMA_ENOTSUP,
	             "velocity solver: slice sides must be in [4, 1024] with prime factors <= 64");
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
	{
		const int nseg = std::max(nx * fw_pieces(nx, ny - 2), ny * fw_pieces(ny, nx - 2));
		const size_t fw_smem = sizeof(SegWalk) * std::max(nseg, 1) +
		                       sizeof(T) * (kFwThreads / 32) * 32 * kFwTile;
		ARMA_CUDA_TRY(cudaFuncSetAttribute(factor_waves_kernel<T>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(fw_smem)));
		factor_waves_kernel<T><<<2 * ns, kFwThreads, fw_smem, c->stream>>>(d_sl, nx, ny, d_k);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
	if (sizeof(T) == sizeof(float) && n2 <= kFuseMax) {
		const size_t smem = sizeof(float2) * (size_t(nx) * (ny + 1) + nx + ny) + sizeof(int) * (nx + ny);
		ARMA_CUDA_TRY(cudaFuncSetAttribute(velocity_fused_kernel,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		float2* spectra =
		    nz > 1 ? static_cast<float2*>(scratch_take(c, sizeof(float2) * n2 * ns)) : nullptr;
		velocity_fused_kernel<<<ns, kFuseThreads, smem, c->stream>>>(
		    reinterpret_cast<const VelSlice<float>*>(d_sl), int(nx), int(ny), px, py, d_k, d_z, nz,
		    depth, spectra);
		ARMA_CUDA_TRY(cudaGetLastError());
		c->launches += 1;
		return;
	}
	// passes of at most ~512 MB of complex work buffers
	const long long per_slice = (long long)sizeof(typename C2<T>::type) * n2 * (1 + nz);
	const int pass = int(std::max<long long>(1, std::min<long long>(ns, (512ll << 20) / per_slice)));
	for (int s0 = 0; s0 < ns; s0 += pass) {
		const ScratchMark mark = scratch_mark(c);
		velocity_general<T>(c, d_sl + s0, std::min(pass, ns - s0), nx, ny, px, py, d_k + 4 * s0, d_z,
		                    nz, depth);
		scratch_release(c, mark);
	}
}

}  // namespace

bool velocity_supported(int nx, int ny) {
	FftPlan p;
	return nx >= 4 && ny >= 4 && nx <= 1024 && ny <= 1024 && make_plan(nx, &p) && make_plan(ny, &p);
}

void launch_velocity_linear(Ctx* c, const void* d_zeta, const int shape[3], int precision,
                            const double delta[3], double depth, const double* z, int nz,
                            const int* t_idx, int ntd, void* d_out, int mode) {
	VelocitySurface v{d_zeta, d_out, shape[0], t_idx, ntd, delta[0], mode, delta[1], delta[2]};
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
				                              v[k].nt, v[k].t_idx[i], v[k].dt, v[k].mode, v[k].dx,
				                              v[k].dy});
		velocity_slices<double>(c, sl, nx, ny, depth, z, nz);
	} else {
		std::vector<VelSlice<float>> sl;
		for (int k = 0; k < n; ++k)
			for (int i = 0; i < v[k].ntd; ++i)
				sl.push_back(VelSlice<float>{static_cast<const float*>(v[k].zeta),
				                             static_cast<float*>(v[k].out) + (long long)i * nz * n2,
				                             v[k].nt, v[k].t_idx[i], v[k].dt, v[k].mode, v[k].dx,
				                             v[k].dy});
		velocity_slices<float>(c, sl, nx, ny, depth, z, nz);
	}
}

}  // namespace armab
