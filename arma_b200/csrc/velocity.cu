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

#include <cooperative_groups.h>

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
// Which slices the derivative reads (offsets from the point in units of
// elements, all uniform over a slice) and which of the four forms applies.
struct ZtTaps {
	int form;  // 0: the slice itself, 1: first slice, 2: last slice, 3: central
	int n;     // slices read
	long long o[3];
};

template <class T>
__device__ __forceinline__ ZtTaps zt_taps(const VelSlice<T>& s, long long n2) {
	const long long d = s.d;
	const int nt = s.nt;
	if (nt - 1 < 2) return ZtTaps{0, 1, {d * n2, 0, 0}};
	if (d == 0) return ZtTaps{1, 3, {2 * n2, n2, 0}};
	if (d == nt - 1) return ZtTaps{2, 3, {d * n2, (d - 1) * n2, (d - 2) * n2}};
	return ZtTaps{3, 2, {(d + 1) * n2, (d - 1) * n2, 0}};
}

// -d zeta/dt from the values v[k] at the offsets o[k]
__device__ __forceinline__ double zt_value(const ZtTaps& k, const double* v, double dt) {
	double r;
	if (k.form == 0) return -v[0];
	if (k.form == 1) r = 0.5 * (-v[0] + 4.0 * v[1] - 3.0 * v[2]);
	else if (k.form == 2) r = 0.5 * (3.0 * v[0] - 4.0 * v[1] + v[2]);
	else r = 0.5 * (v[0] - v[1]);
	if (dt != 1.0) r /= dt;  // a division by 1 is exact: skipped
	return -r;
}

template <class T>
__device__ __forceinline__ double zeta_t(const VelSlice<T>& s, long long n2, long long p) {
	const T* f = s.zeta + p;
	const ZtTaps k = zt_taps(s, n2);
	double v[3] = {0.0, 0.0, 0.0};
	for (int q = 0; q < k.n; ++q) v[q] = double(f[k.o[q]]);
	return zt_value(k, v, s.dt);
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
// staging tiles of 32 x kFwTile elements per warp: two in FP32 (the next 32
// positions stage while the current ones are walked), one in FP64 (two would
// halve the CTAs per SM)
template <class T>
constexpr int fw_tiles() { return sizeof(T) == 4 ? 2 : 1; }

// One element from global into shared memory, asynchronously (L1-allocating
// cp.async of 4 or 8 bytes); cp_async_commit closes a group of them and
// cp_async_wait<N> waits until at most N of this thread's groups are pending.
template <class T>
__device__ __forceinline__ void cp_async_elem(T* dst_smem, const T* src) {
	static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
	const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst_smem));
	asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(sizeof(T))
	             : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
	asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

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
	// |period difference| extremes of the pairs (r-1, r) with r >= 2 that
	// closed; k is a decreasing function of it, evaluated once at the end
	double dmin = INFINITY, dmax = -INFINITY;
};

// The reference forms k = (2 pi / |2 (p1 - p0)|)^2 / g for every pair and
// keeps min and max k.  Rounded division, squaring and division by g are each
// monotone, so k is a non-increasing function of d = |p1 - p0| and
// min k = k(max d), max k = k(min d) exactly; the walk keeps d's extremes and
// k_of is applied once per axis.  (A NaN period gives a NaN d and a NaN k,
// which the reference's comparisons skip; so do these.)
__device__ __forceinline__ void pair_k(double p0, double p1, double& dmin, double& dmax) {
	const double d = fabs(p1 - p0);
	if (d < dmin) dmin = d;
	if (d > dmax) dmax = d;
}

__device__ __forceinline__ double k_of(double d) {
	const double w = k2Pi / fabs(d * 2.0);
	return w * w / kG;
}

// The next position of a thread's own segment, in loop order, when `ev` (it
// is an extremum) with elevation e and period p: the first event opens run 0;
// an event of the open run's sign replaces its representative only when its
// |elevation| is larger (the first maximum stays); an event of the other sign
// closes the open run (run 0 and run 1 keep their representatives for a later
// join, every later run adds its pair with the run before) and opens the next.
// Written as selects rather than branches, so that the lanes of a warp, each
// walking its own line, do not diverge on the event's kind.
__device__ __forceinline__ void seg_event_if(SegWalk& st, bool ev, double e, double p) {
	const int s = e > 0.0 ? 1 : 0;
	const double ae = fabs(e);
	const bool first = ev && st.m == 0;
	const bool same = ev && st.m != 0 && s == st.open.sign;
	const bool close = ev && st.m != 0 && s != st.open.sign;
	const bool better = same && st.open.best_e < ae;
	const int r = st.m - 1;
	const bool c0 = close && r == 0, c1 = close && r == 1, pk = close && r >= 2;
	st.r0.sign = c0 ? st.open.sign : st.r0.sign;
	st.r0.best_e = c0 ? st.open.best_e : st.r0.best_e;
	st.r0.best_p = c0 ? st.open.best_p : st.r0.best_p;
	st.r1_p = c1 ? st.open.best_p : st.r1_p;
	// pair_k: comparisons with a NaN difference are false and change nothing
	const double d = fabs(st.open.best_p - st.prev_p);
	st.dmin = pk && d < st.dmin ? d : st.dmin;
	st.dmax = pk && d > st.dmax ? d : st.dmax;
	st.prev_p = close ? st.open.best_p : st.prev_p;
	const bool take = first || close || better;
	st.open.best_e = take ? ae : st.open.best_e;
	st.open.best_p = take ? p : st.open.best_p;
	st.open.sign = (first || close) ? s : st.open.sign;
	st.m += (first || close) ? 1 : 0;
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
	C.dmin = fmin(A.dmin, B.dmin);
	C.dmax = fmax(A.dmax, B.dmax);
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
		else pair_k(A.prev_p, R.best_p, C.dmin, C.dmax);
		if (B.m >= 3) {  // B's run 1 (index rR + 1) closed
			if (rR == 0) C.r1_p = B.r1_p;
			else pair_k(R.best_p, B.r1_p, C.dmin, C.dmax);
		}
		C.open = B.open;
		C.prev_p = B.m == 2 ? R.best_p : B.prev_p;
		return C;
	}
	const int rA = A.m - 1;  // A's open run closes
	C.m = A.m + B.m;
	if (rA == 0) C.r0 = A.open;
	else if (rA == 1) C.r1_p = A.open.best_p;
	else pair_k(A.prev_p, A.open.best_p, C.dmin, C.dmax);
	if (B.m == 1) {
		C.open = B.open;
		C.prev_p = A.open.best_p;
		return C;
	}
	if (A.m == 1) C.r1_p = b0.best_p;  // B's run 0 (index A.m) closed
	else pair_k(A.open.best_p, b0.best_p, C.dmin, C.dmax);
	if (B.m >= 3) pair_k(b0.best_p, B.r1_p, C.dmin, C.dmax);  // index A.m + 1 >= 2
	C.open = B.open;
	C.prev_p = B.m == 2 ? b0.best_p : B.prev_p;
	return C;
}

// Segment summaries in shared memory as a structure of arrays (8 double and
// 3 int arrays of nseg entries), so that neighbouring threads touch
// neighbouring words.
constexpr int kSegBytes = 8 * 8 + 3 * 4;
// bytes of n summaries, rounded up to 16 so that the staging tile after them
// is aligned for any element type
__host__ __device__ inline size_t seg_region_bytes(int n) {
	return (size_t(kSegBytes) * size_t(n) + 15) & ~size_t(15);
}

struct SegStore {
	double *oe, *op, *prev, *r0e, *r0p, *r1p, *dmin, *dmax;
	int *m, *osign, *r0s;
	__device__ SegStore(unsigned char* base, int n) {
		double* d = reinterpret_cast<double*>(base);
		oe = d; op = d + n; prev = d + 2 * n; r0e = d + 3 * n; r0p = d + 4 * n; r1p = d + 5 * n;
		dmin = d + 6 * n; dmax = d + 7 * n;
		int* q = reinterpret_cast<int*>(d + 8 * n);
		m = q; osign = q + n; r0s = q + 2 * n;
	}
	__device__ void put(int i, const SegWalk& w) const {
		oe[i] = w.open.best_e; op[i] = w.open.best_p; prev[i] = w.prev_p;
		r0e[i] = w.r0.best_e; r0p[i] = w.r0.best_p; r1p[i] = w.r1_p;
		dmin[i] = w.dmin; dmax[i] = w.dmax;
		m[i] = w.m; osign[i] = w.open.sign; r0s[i] = w.r0.sign;
	}
	__device__ SegWalk get(int i) const {
		SegWalk w;
		w.open = Run{osign[i], oe[i], op[i]};
		w.r0 = Run{r0s[i], r0e[i], r0p[i]};
		w.prev_p = prev[i]; w.r1_p = r1p[i]; w.dmin = dmin[i]; w.dmax = dmax[i]; w.m = m[i];
		return w;
	}
};

__device__ __forceinline__ SegWalk seg_shfl_down(const SegWalk& w, int d) {
	SegWalk o;
	o.m = __shfl_down_sync(0xffffffffu, w.m, d);
	o.open.sign = __shfl_down_sync(0xffffffffu, w.open.sign, d);
	o.open.best_e = __shfl_down_sync(0xffffffffu, w.open.best_e, d);
	o.open.best_p = __shfl_down_sync(0xffffffffu, w.open.best_p, d);
	o.prev_p = __shfl_down_sync(0xffffffffu, w.prev_p, d);
	o.r0.sign = __shfl_down_sync(0xffffffffu, w.r0.sign, d);
	o.r0.best_e = __shfl_down_sync(0xffffffffu, w.r0.best_e, d);
	o.r0.best_p = __shfl_down_sync(0xffffffffu, w.r0.best_p, d);
	o.r1_p = __shfl_down_sync(0xffffffffu, w.r1_p, d);
	o.dmin = __shfl_down_sync(0xffffffffu, w.dmin, d);
	o.dmax = __shfl_down_sync(0xffffffffu, w.dmax, d);
	return o;
}

// Extremum test and quadratic vertex at position a of a line (z0 = z(a),
// z1 = z(a-1), z2 = z(a+1)).  The test needs only the signs of z0 - z1 and
// z0 - z2, which a rounded subtraction always gets right, so it runs in the
// input's own precision; the vertex (the reference's formula) is FP64.
template <class T>
__device__ __forceinline__ bool fw_extremum(T z0, T z1, T z2) {
	return (z0 - z1 > T(0)) == (z0 - z2 > T(0));
}

template <class T>
__device__ __forceinline__ void fw_vertex(T z0, T z1, T z2, double dt, int t, double& elev,
                                          double& tex) {
	const double dw1 = double(z0) - double(z1), dw2 = double(z0) - double(z2);
	double aa, bb, cc;
	if (dt == 1.0) {  // x / 1 and x * 1 are exact: the same values without two divisions
		aa = -0.5 * (dw1 + dw2);
		bb = dw1 - aa * (2.0 * t - 1.0);
		cc = double(z0) - t * (aa * t + bb);
	} else {
		aa = -0.5 * (dw1 + dw2) / (dt * dt);
		bb = dw1 / dt - aa * dt * (2.0 * t - 1.0);
		cc = double(z0) - t * dt * (aa * t * dt + bb);
	}
	tex = -0.5 * bb / aa;
	elev = cc + tex * (bb + aa * tex);
}

// n (<= kFwBatch) consecutive positions after (z1, z0), es elements apart
// from zn on, fed to the walk in order; leaves (z1, z0) at the last two values.  The vertices of kFwIlp
// positions are computed before any is fed to the walk, extremum or not, so
// that their FP64 chains (a division each) run side by side: a warp takes the
// vertex path whenever any of its lanes has an extremum, which is nearly
// always, so computing it for every position costs the warp nothing more.
constexpr int kFwBatch = 8;
constexpr int kFwIlp = 4;
template <class T>
__device__ __forceinline__ void fw_batch(SegWalk& st, T& z1, T& z0, const T* zn, int es, int n,
                                         double dt, int t) {
#pragma unroll
	for (int k0 = 0; k0 < kFwBatch; k0 += kFwIlp) {
		double e[kFwIlp], p[kFwIlp];
		bool ev[kFwIlp];
#pragma unroll
		for (int k = 0; k < kFwIlp; ++k) {
			const T z2 = k0 + k < n ? zn[(k0 + k) * es] : z0;
			ev[k] = k0 + k < n && fw_extremum(z0, z1, z2);
			fw_vertex(z0, z1, z2, dt, t, e[k], p[k]);
			if (k0 + k < n) {
				z1 = z0;
				z0 = z2;
			}
		}
#pragma unroll
		for (int k = 0; k < kFwIlp; ++k) seg_event_if(st, ev[k], e[k], p[k]);
	}
}

// Pieces per line for a launch of ns slices: a work unit is one piece of 32
// neighbouring lines, walked by one warp.  As few pieces as keep two waves of
// units (16 warps per SM) in the launch, at least 8 positions each and no
// more than two units per warp of a full CTA (which bounds the segments'
// shared memory): long units keep the next positions staging while a warp
// walks (a unit of one chunk waits for its loads) and leave fewer segments
// to join.
inline int fw_piece_cap(int outer, int npos) {
	const int blocks = (outer + 31) / 32;
	return npos < 16 ? 1 : std::min(npos / 8, (2 * (kFwThreads / 32) + blocks - 1) / blocks);
}
inline int fw_pieces(int outer, int npos, int ns, int num_sms) {
	const long long units1 = 2ll * ns * ((outer + 31) / 32);  // both axes' CTAs, one piece each
	const long long want = 2ll * 16 * num_sms;
	const long long p = (want + units1 - 1) / units1;
	return int(std::max(1ll, std::min<long long>(p, fw_piece_cap(outer, npos))));
}

// One CTA per (slice, axis).  axis 0 loops y outer, x inner over z(x,y): lane
// b walks column y = b down x; axis 1 (the reference's transposed call) x
// outer, y inner: lane b walks row x = b.  Each warp stages 34 positions of
// its 32 lines at a time into shared memory with asynchronous copies (rows of
// the slice, coalesced), in FP32 into two tiles so that the next positions
// arrive while the current ones are walked; both passes then run the same
// walk.  Writes min_k, max_k of the axis.
template <class T>
__global__ void __launch_bounds__(kFwThreads, 2)
factor_waves_kernel(const VelSlice<T>* __restrict__ sl, int nx, int ny, int pieces0, int pieces1,
                    double* __restrict__ kout) {
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
	const int P = axis == 0 ? pieces0 : pieces1, per = (npos + P - 1) / P;
	const int nseg = outer * P, blocks = (outer + 31) / 32;
	// segments, then the warps' results: the larger axis's count for both
	const int nstore = max(max(ny * pieces0, nx * pieces1), nwarps);
	const SegStore seg(fw_smem, nstore);
	T* tile = reinterpret_cast<T*>(fw_smem + seg_region_bytes(nstore)) +
	          warp * fw_tiles<T>() * 32 * kFwTile;
	for (int u = warp; u < blocks * P; u += nwarps) {
		const int piece = u / blocks, b0 = (u % blocks) * 32, b = b0 + lane;
		const int a_lo = 1 + piece * per, a_hi = 1 + min(npos, (piece + 1) * per);  // [a_lo, a_hi)
		SegWalk st;
		const int lines = min(32, outer - b0);
		// positions c0-1 .. c0+32 of the unit's lines (those inside the
		// slice) into tile tb, as one group of asynchronous copies: for the x
		// pass (lines are columns) 34 rows of 32 lines, coalesced along the
		// rows; for the y pass (lines are rows) 32 lines of 34 positions at a
		// row pitch of kFwTile
		auto stage = [&](int c0, T* tb) {
			if (axis == 0) {
				if (lane < lines)
					for (int r = 0; r < 34 && c0 - 1 + r < nx; ++r)
						cp_async_elem(tb + r * 32 + lane, z + (long long)(c0 - 1 + r) * ny + b0 + lane);
			} else {
				for (int r = 0; r < lines; ++r) {
					const T* zr = z + (long long)(b0 + r) * ny;
					if (c0 - 1 + lane < ny) cp_async_elem(tb + r * kFwTile + lane, zr + c0 - 1 + lane);
					if (lane < 2 && c0 + 31 + lane < ny)
						cp_async_elem(tb + r * kFwTile + 32 + lane, zr + c0 + 31 + lane);
				}
			}
			cp_async_commit();
		};
		// the lane's line in a tile: position c0 - 1 + k at line[k * es]
		const int loff = axis == 0 ? lane : lane * kFwTile, es = axis == 0 ? 32 : 1;
		constexpr int NB = fw_tiles<T>();
		int cur = 0;
		if (NB == 2 && a_lo < a_hi) stage(a_lo, tile);
		for (int c0 = a_lo; c0 < a_hi; c0 += 32) {
			T* tb = tile + cur * 32 * kFwTile;
			if (NB == 2 && c0 + 32 < a_hi) {
				// the other tile was last read in the previous step, which ended
				// with a warp barrier
				stage(c0 + 32, tile + (cur ^ 1) * 32 * kFwTile);
				cp_async_wait<1>();
			} else {
				if (NB == 1) stage(c0, tb);
				cp_async_wait<0>();
			}
			__syncwarp();
			if (b < outer) {
				const T* line = tb + loff;
				T z1 = line[0], z0 = line[es];
				const int n = min(32, a_hi - c0);
				for (int k0 = 0; k0 < n; k0 += kFwBatch)
					fw_batch(st, z1, z0, line + (2 + k0) * es, es, min(kFwBatch, n - k0), dt, t);
			}
			__syncwarp();  // tile tb read by every lane before it is staged again
			cur ^= NB - 1;
		}
		if (b < outer) seg.put(b * P + piece, st);  // loop order: line, then piece
	}
	__syncthreads();
	// join in loop order: every warp a contiguous range, every lane a
	// contiguous piece of it folded in sequence, then a shuffle tree over the
	// lanes (lane l's range precedes lane l + d's), then the warps' results
	const int per_warp = (nseg + nwarps - 1) / nwarps;
	const int lo = min(nseg, warp * per_warp), hi = min(nseg, lo + per_warp);
	const int per_lane = (hi - lo + 31) / 32;
	SegWalk acc;
	for (int j = 0; j < per_lane; ++j) {
		const int i = lo + lane * per_lane + j;
		if (i < hi) acc = seg_join(acc, seg.get(i));
	}
	for (int d = 1; d < 32; d <<= 1) {
		const SegWalk other = seg_shfl_down(acc, d);
		if ((lane & (2 * d - 1)) == 0) acc = seg_join(acc, other);
	}
	__syncthreads();  // the segment arrays are read; warp results reuse them
	if (lane == 0) seg.put(warp, acc);
	__syncthreads();
	if (threadIdx.x == 0) {
		SegWalk all;
		for (int w = 0; w < nwarps; ++w) all = seg_join(all, seg.get(w));
		if (all.m >= 3) pair_k(all.r0.best_p, all.r1_p, all.dmin, all.dmax);  // runs 0 and 1
		// min k and max k, starting from DBL_MAX and DBL_MIN as the reference does
		const bool any = all.dmax >= 0.0;
		kout[slice * 4 + axis] = any ? fmin(DBL_MAX, k_of(all.dmax)) : DBL_MAX;
		kout[slice * 4 + 2 + axis] = any ? fmax(DBL_MIN, k_of(all.dmin)) : DBL_MIN;
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
	const double s2 = u * u + v * v;
	if (z == 0.0 && h == INFINITY && s2 > 0.0 && s2 <= DBL_MAX) {
		// l = 2 pi sqrt(s2) is finite and positive: -l z = -0 (exp = 1) and
		// -2 l h = -inf (exp = 0), so the formula below gives 4 pi 1 / 1
		// without the square root
		return k2Pi * 2.0 * 1.0 / 1.0;
	}
	const double l = k2Pi * sqrt(s2);
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

// ---------------------------------------------------------------- 2c. real fused
// FP32 linear solver (mode 0) on power-of-two slices of up to 32768 points.
//
// zeta_t is real and only Re of the inverse is kept (the reference keeps the
// real part, src/velocity/linear_solver.cc:115), so with F = FFT2(zeta_t)
// Hermitian,  Re IFFT2(W F) = IFFT2(We F),  We(k) = (W(k) + W(-k)) / 2,  and
// We F is Hermitian again.  Rows are paired: z(p, y) = u(2p, y) + i u(2p+1, y)
// (u = zeta_t) is an M x ny complex array, M = nx / 2, whose FFT2 Z gives the
// spectra E, O of the even and odd rows,
//     E(a, b) = (Z(a, b) + conj Z(-a, -b)) / 2,  O = (Z - conj Z(-a, -b)) / 2i,
//     U(a, b) = E + W_nx^a O,  U(a + M, b) = E - W_nx^a O.
// The filtered spectrum U' = We U is packed back the same way,
//     E' = S E + D W_nx^a O,  O' = S O + D W_nx^-a E,   S, D = (We(a) +- We(a+M)) / 2,
// Z'(a, b) = E' + i O' and Z'(-a, -b) = conj E' + i conj O', and the inverse FFT2
// of Z' holds M ny (phi(2p, y) + i phi(2p+1, y)).  One CTA per slice holds the
// M x ny array in shared memory (half of a full complex spectrum); the line
// FFTs run in registers.
//
// Line FFT (forward, natural order in and out; the inverse conjugates):
// N = R1 R2 points by T = N / 16 threads of one warp, 16 points per thread.
//   step 1: for n2 (thread t, t + T, ...): v[n1] = x[R2 n1 + n2], R1-point DFT,
//           v[k1] *= W_N^(n2 k1)
//   exchange through the line's own storage: x[R2 k1 + n2] = v[k1]
//   step 2: for k1 (thread t, t + T, ...): w[n2] = x[R2 k1 + n2], R2-point DFT,
//           X[k1 + R1 k2] = w[k2]
// The threads of a line are consecutive lanes of one warp, so the exchange
// needs only __syncwarp.
constexpr int kRealMaxPoints = 32768;  // nx * ny of the real fused path (128 KB of float2)

template <bool INV>
__device__ __forceinline__ float2 cmul_tw(float2 a, float2 w) {
	// a * w (forward) or a * conj(w) (inverse)
	return INV ? make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y)
	           : make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// t * (-i) forward, t * i inverse
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 t) {
	return INV ? make_float2(-t.y, t.x) : make_float2(t.y, -t.x);
}

template <bool INV>
__device__ __forceinline__ void dft4r(float2& a, float2& b, float2& c, float2& d) {
	const float2 s0 = make_float2(a.x + c.x, a.y + c.y), d0 = make_float2(a.x - c.x, a.y - c.y);
	const float2 s1 = make_float2(b.x + d.x, b.y + d.y);
	const float2 d1 = mul_mi<INV>(make_float2(b.x - d.x, b.y - d.y));
	a = make_float2(s0.x + s1.x, s0.y + s1.y);
	b = make_float2(d0.x + d1.x, d0.y + d1.y);
	c = make_float2(s0.x - s1.x, s0.y - s1.y);
	d = make_float2(d0.x - d1.x, d0.y - d1.y);
}

// W_16^j, j = 0..15 (exp(-2 pi i j / 16)): the roots of the 16-point DFT
__device__ __forceinline__ float2 w16(int j) {
	constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
	constexpr float h = 0.70710678118654752440f;
	switch (j & 15) {
		case 0: return make_float2(1.f, 0.f);
		case 1: return make_float2(c1, -s1);
		case 2: return make_float2(h, -h);
		case 3: return make_float2(s1, -c1);
		case 4: return make_float2(0.f, -1.f);
		case 5: return make_float2(-s1, -c1);
		case 6: return make_float2(-h, -h);
		case 7: return make_float2(-c1, -s1);
		case 8: return make_float2(-1.f, 0.f);
		case 9: return make_float2(-c1, s1);
		case 10: return make_float2(-h, h);
		case 11: return make_float2(-s1, c1);
		case 12: return make_float2(0.f, 1.f);
		case 13: return make_float2(s1, c1);
		case 14: return make_float2(h, h);
		default: return make_float2(c1, s1);
	}
}

// In-register R-point DFT of v[0..R), natural order out.
template <int R, bool INV>
__device__ __forceinline__ void dft_reg(float2* v) {
	if constexpr (R == 1) {
	} else if constexpr (R == 2) {
		const float2 a = v[0], b = v[1];
		v[0] = make_float2(a.x + b.x, a.y + b.y);
		v[1] = make_float2(a.x - b.x, a.y - b.y);
	} else if constexpr (R == 4) {
		dft4r<INV>(v[0], v[1], v[2], v[3]);
	} else if constexpr (R == 8) {
		// radix 2 over two 4-point DFTs of the even and odd samples
		float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
		float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
		dft4r<INV>(e0, e1, e2, e3);
		dft4r<INV>(o0, o1, o2, o3);
		float2 e[4] = {e0, e1, e2, e3}, o[4] = {o0, o1, o2, o3};
#pragma unroll
		for (int k = 0; k < 4; ++k) {
			const float2 t = cmul_tw<INV>(o[k], w16(2 * k));
			v[k] = make_float2(e[k].x + t.x, e[k].y + t.y);
			v[k + 4] = make_float2(e[k].x - t.x, e[k].y - t.y);
		}
	} else if constexpr (R == 16) {
		// radix 4: F_r = DFT4(v[r], v[r+4], v[r+8], v[r+12]), then per k1 a
		// DFT4 over r of W_16^(r k1) F_r[k1] -> X[k1 + 4 k2]
		float2 f[4][4];
#pragma unroll
		for (int r = 0; r < 4; ++r) {
			f[r][0] = v[r];
			f[r][1] = v[r + 4];
			f[r][2] = v[r + 8];
			f[r][3] = v[r + 12];
			dft4r<INV>(f[r][0], f[r][1], f[r][2], f[r][3]);
		}
#pragma unroll
		for (int k1 = 0; k1 < 4; ++k1) {
			float2 a = f[0][k1];
			float2 b = cmul_tw<INV>(f[1][k1], w16(k1));
			float2 c = cmul_tw<INV>(f[2][k1], w16(2 * k1));
			float2 d = cmul_tw<INV>(f[3][k1], w16(3 * k1));
			dft4r<INV>(a, b, c, d);
			v[k1] = a;
			v[k1 + 4] = b;
			v[k1 + 8] = c;
			v[k1 + 12] = d;
		}
	}
}

template <int N> struct LineShape;
template <> struct LineShape<16> { static constexpr int R1 = 16, R2 = 1; };
template <> struct LineShape<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct LineShape<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct LineShape<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct LineShape<256> { static constexpr int R1 = 16, R2 = 16; };

// N-point FFT of the line x[0], x[es], ... by thread t of its T = N / 16
// threads.  tw[j * ts] = W_N^j.  Every lane of the warp must call it the same
// number of times (the exchange synchronises the warp); `active` = false for
// lanes without a line.
template <int N, bool INV>
__device__ __forceinline__ void line_fft(float2* x, int es, int t, const float2* tw, int ts,
                                         bool active) {
	constexpr int R1 = LineShape<N>::R1, R2 = LineShape<N>::R2, T = N / 16;
	if constexpr (R2 == 1) {
		float2 v[16];
		if (active) {
#pragma unroll
			for (int k = 0; k < 16; ++k) v[k] = x[k * es];
			dft_reg<16, INV>(v);
#pragma unroll
			for (int k = 0; k < 16; ++k) x[k * es] = v[k];
		}
		return;
	} else {
		// The exchange position of (k1, n2) is R2 k1 + (n2 + k1) mod R2: a
		// rotation inside each block of R2, which spreads the step-2 reads of
		// neighbouring threads over the banks.  The rotated positions were
		// loaded by other threads in step 1, so every load of the line
		// completes (warp barrier) before any exchange write.
		constexpr int S1 = R2 / T, S2 = R1 / T;
		float2 v[S1][R1];
		if (active) {
#pragma unroll
			for (int s = 0; s < S1; ++s) {
				const int n2 = t + T * s;
#pragma unroll
				for (int n1 = 0; n1 < R1; ++n1) v[s][n1] = x[(R2 * n1 + n2) * es];
				dft_reg<R1, INV>(v[s]);
#pragma unroll
				for (int k1 = 1; k1 < R1; ++k1) v[s][k1] = cmul_tw<INV>(v[s][k1], tw[n2 * k1 * ts]);
			}
		}
		__syncwarp();
		if (active) {
#pragma unroll
			for (int s = 0; s < S1; ++s) {
				const int n2 = t + T * s;
#pragma unroll
				for (int k1 = 0; k1 < R1; ++k1) x[(R2 * k1 + (n2 + k1) % R2) * es] = v[s][k1];
			}
		}
		__syncwarp();
		float2 w[S2][R2];
		if (active) {
#pragma unroll
			for (int s = 0; s < S2; ++s) {
				const int k1 = t + T * s;
#pragma unroll
				for (int n2 = 0; n2 < R2; ++n2) w[s][n2] = x[(R2 * k1 + (n2 + k1) % R2) * es];
				dft_reg<R2, INV>(w[s]);
			}
		}
		__syncwarp();
		if (active) {
#pragma unroll
			for (int s = 0; s < S2; ++s) {
				const int k1 = t + T * s;
#pragma unroll
				for (int k2 = 0; k2 < R2; ++k2) x[(k1 + R1 * k2) * es] = w[s][k2];
			}
		}
	}
}

// FFTs of `nlines` lines of length N: line l at a + l * lstride, elements
// es apart.  Each line gets T = N / 16 lanes of one warp: consecutive lanes
// on one line (rows), or, with lines_fastest, consecutive lanes on
// consecutive lines (columns, whose elements are a row stride apart).  Every
// warp runs the same number of rounds.
template <int N, bool INV, int NT, bool LINES_FASTEST>
__device__ __forceinline__ void lines_fft(float2* a, int nlines, int lstride, int es,
                                          const float2* tw, int ts) {
	constexpr int T = N / 16, G = 32 / T;  // G lines per warp
	constexpr int per_round = NT / T;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int g = warp * G + (LINES_FASTEST ? lane % G : lane / T);
	const int t = LINES_FASTEST ? lane / G : lane % T;
	for (int l0 = 0; l0 < nlines; l0 += per_round) {
		const int l = l0 + g;
		const bool active = l < nlines;
		line_fft<N, INV>(a + (active ? l : 0) * lstride, es, t, tw, ts, active);
	}
	__syncwarp();
}

// Row stride of the M x NY array in float2, chosen by counting the bank
// conflicts of every access of the row and column passes (64-bit accesses,
// 16 banks of 8 bytes per half warp): NY + NY / 16 keeps the row passes free
// of conflicts; the column passes of M >= 64 keep at most two-way conflicts.
template <int M, int NY> struct RealLd {
	static constexpr int v = NY == 16 ? 17 : NY == 256 ? (M >= 64 ? 264 : 256) : NY + NY / 16;
};

// Even part of the window at natural-order frequency (kx, ky):
// (W(k) + W(-k)) / 2 with W evaluated at the rotated grid indices.  Not
// inlined: the FP64 window code would otherwise hold registers across the
// FFT kernel's pairing loop.
__device__ __noinline__ double window_even(int kx, int ky, int nx, int ny, double dkx, double dky,
                                           double z, double depth) {
	const int mx = kx == 0 ? 0 : nx - kx, my = ky == 0 ? 0 : ny - ky;
	const double w1 = window_fixed(rotate_src(kx, nx), rotate_src(ky, ny), nx, ny, dkx, dky, z, depth);
	const double w2 = window_fixed(rotate_src(mx, nx), rotate_src(my, ny), nx, ny, dkx, dky, z, depth);
	return 0.5 * (w1 + w2);
}

// True when every entry of the fixed window is the same 4 pi: z = 0 at
// infinite depth with s2 = (dkx i)^2 + (dky j)^2 positive and finite at every
// (i, j) != (0, 0) of the nx x ny grid.  Rounding keeps s2 monotone in i and
// j, so (1, 0), (0, 1) and (nx-1, ny-1) decide it; window_raw then returns its
// z = 0 shortcut everywhere, (0, 0) copies (1, 1) and no edge fix applies, so
// the even part is that constant and its odd part 0.
__device__ __forceinline__ bool window_flat(int nx, int ny, double dkx, double dky, double z,
                                            double depth) {
	if (!(z == 0.0 && depth == INFINITY)) return false;
	const double ex = dkx * (nx - 1), ey = dky * (ny - 1);
	return dkx * dkx > 0.0 && dky * dky > 0.0 && ex * ex + ey * ey <= DBL_MAX;
}
// the value of that window, as window_raw forms it
__device__ __forceinline__ double window_flat_value() { return k2Pi * 2.0 * 1.0 / 1.0; }

// The solver's input of rows 2p and 2p + 1 (p = p0 + i, i < rows) into
// A[i * LD + y] as (row 2p, row 2p + 1).  The linear solver's -zeta_t loads
// the slices of kRealBatch points of each thread before forming any of them,
// so that a thread has that many loads in flight; the high-amplitude input
// goes point by point.
constexpr int kRealBatch = 8;
template <int NY, int NT, int LD>
__device__ __forceinline__ void real_input_rows(const VelSlice<float>& S, int NX, int p0, int rows,
                                                float2* A) {
	const long long n2 = (long long)NX * NY;
	const int total = rows * NY;
	if (S.mode != 0) {
		for (int q = threadIdx.x; q < total; q += NT) {
			const int i = q / NY, y = q % NY, p = p0 + i;
			double re, im;
			solver_input(S, NX, NY, (long long)(2 * p) * NY + y, re, im);
			const double r0 = re;
			solver_input(S, NX, NY, (long long)(2 * p + 1) * NY + y, re, im);
			A[i * LD + y] = make_float2(float(r0), float(re));
		}
		return;
	}
	const ZtTaps k = zt_taps(S, n2);
	for (int q0 = threadIdx.x; q0 < total; q0 += kRealBatch * NT) {
		float v[kRealBatch][2][3];
#pragma unroll
		for (int u = 0; u < kRealBatch; ++u) {
			const int q = q0 + u * NT;
			if (q < total) {
				const int i = q / NY, y = q % NY;
				const float* f = S.zeta + (long long)(2 * (p0 + i)) * NY + y;
#pragma unroll
				for (int h = 0; h < 2; ++h)
#pragma unroll
					for (int j = 0; j < 3; ++j)
						if (j < k.n) v[u][h][j] = f[h * NY + k.o[j]];
			}
		}
#pragma unroll
		for (int u = 0; u < kRealBatch; ++u) {
			const int q = q0 + u * NT;
			if (q < total) {
				const int i = q / NY, y = q % NY;
				double a[3], b[3];
#pragma unroll
				for (int j = 0; j < 3; ++j) {
					a[j] = j < k.n ? double(v[u][0][j]) : 0.0;
					b[j] = j < k.n ? double(v[u][1][j]) : 0.0;
				}
				A[i * LD + y] = make_float2(float(zt_value(k, a, S.dt)), float(zt_value(k, b, S.dt)));
			}
		}
	}
}

template <int M, int NY, int NT>
__global__ void __launch_bounds__(NT, NT == 256 ? 2 : 1)
velocity_real_kernel(const VelSlice<float>* __restrict__ sl, const double* __restrict__ kinfo,
                     const double* __restrict__ zs, int nz, double depth,
                     float2* __restrict__ spectra) {
	constexpr int NX = 2 * M, LD = RealLd<M, NY>::v;
	constexpr int L = NX > NY ? NX : NY;  // twiddle table: W_L^j
	extern __shared__ __align__(16) unsigned char smem_raw[];
	float2* A = reinterpret_cast<float2*>(smem_raw);  // M rows of LD
	float2* tw = A + M * LD;                           // L
	const int s = blockIdx.x;
	const VelSlice<float> S = sl[s];
	constexpr int n2 = NX * NY;
	for (int j = threadIdx.x; j < L; j += NT) {
		double sn, cs;
		sincospi(2.0 * j / L, &sn, &cs);
		tw[j] = make_float2(float(cs), float(-sn));
	}
	// zeta_t of rows 2p and 2p + 1 into z(p, y)
	real_input_rows<NY, NT, LD>(S, NX, 0, M, A);
	__syncthreads();
	lines_fft<NY, false, NT, false>(A, M, LD, 1, tw, L / NY);  // rows
	__syncthreads();
	lines_fft<M, false, NT, true>(A, NY, 1, LD, tw, L / M);    // columns
	__syncthreads();
	float2* spec = spectra ? spectra + (long long)s * M * NY : nullptr;
	if (spec) {
		for (int q = threadIdx.x; q < M * NY; q += NT) spec[q] = A[(q / NY) * LD + q % NY];
		__syncthreads();  // the pairing pass rewrites A
	}
	const double wx = 1.0 / kinfo[s * 4 + 0], wy = 1.0 / kinfo[s * 4 + 1];
	const double dkx = wx / (NX - 1), dky = wy / (NY - 1);
	const float inv = float(1.0 / double(M * NY));
	for (int iz = 0; iz < nz; ++iz) {
		if (iz > 0) {
			__syncthreads();  // the previous depth's output read A
			for (int q = threadIdx.x; q < M * NY; q += NT) A[(q / NY) * LD + q % NY] = spec[q];
			__syncthreads();
		}
		const double z = zs[iz];
		auto We = [&](int kx, int ky) {
			return window_even(kx, ky, NX, NY, dkx, dky, z, depth);
		};
		const bool flat = window_flat(NX, NY, dkx, dky, z, depth);
		const float flat_w = float(window_flat_value());
		// one thread per pair {(a, b), (-a, -b)}: b in [0, NY/2], a in [0, M),
		// with b in {0, NY/2} only a <= M/2 (the others are partners);
		// consecutive threads on consecutive b (one row of A)
		for (int q = threadIdx.x; q < M * (NY / 2 + 1); q += NT) {
			const int a = q / (NY / 2 + 1), b = q % (NY / 2 + 1);
			if ((b == 0 || b == NY / 2) && a > M / 2) continue;
			const int am = a == 0 ? 0 : M - a, bm = b == 0 ? 0 : NY - b;
			const float2 z1 = A[a * LD + b], z2 = A[am * LD + bm];
			// E = (z1 + conj z2) / 2, O = (z1 - conj z2) / 2i
			const float2 E = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
			const float2 O = make_float2(0.5f * (z1.y + z2.y), -0.5f * (z1.x - z2.x));
			float2 E2, O2;
			if (flat) {  // S = the constant, D = 0: the same values without the window calls
				E2 = make_float2(flat_w * E.x, flat_w * E.y);
				O2 = make_float2(flat_w * O.x, flat_w * O.y);
			} else {
				const double wa = We(a, b), wb = We(a + M, b);
				const float Sv = float(0.5 * (wa + wb)), Dv = float(0.5 * (wa - wb));
				const float2 w = tw[a * (L / NX)];  // W_nx^a
				const float2 wO = cmul_tw<false>(O, w), wE = cmul_tw<true>(E, w);
				E2 = make_float2(Sv * E.x + Dv * wO.x, Sv * E.y + Dv * wO.y);
				O2 = make_float2(Sv * O.x + Dv * wE.x, Sv * O.y + Dv * wE.y);
			}
			A[a * LD + b] = make_float2(E2.x - O2.y, E2.y + O2.x);     // E' + i O'
			A[am * LD + bm] = make_float2(E2.x + O2.y, -E2.y + O2.x);  // conj E' + i conj O'
		}
		__syncthreads();
		lines_fft<M, true, NT, true>(A, NY, 1, LD, tw, L / M);    // columns
		__syncthreads();
		lines_fft<NY, true, NT, false>(A, M, LD, 1, tw, L / NY);  // rows
		__syncthreads();
		float* out = S.out + (long long)iz * n2;
		auto f = [&](int r, int c) -> double {
			const float2 v = A[(r >> 1) * LD + c];
			return double((r & 1) ? v.y : v.x) * double(inv);
		};
		for (int q = threadIdx.x; q < n2; q += NT) {
			const int x = q / NY, y = q % NY;
			if (x > 0 && y > 0) {
				const float2 v = A[(x >> 1) * LD + y];
				out[q] = ((x & 1) ? v.y : v.x) * inv;
			} else {
				out[q] = float(finish_at(x, y, NX, NY, f));
			}
		}
	}
}

// The instantiated (M, NY) shapes: M in {16, 32, 64, 128}, NY in {16..256},
// M * NY <= 16384.
template <int M, int NY>
bool launch_real_shape(Ctx* c, const VelSlice<float>* d_sl, int ns, int nx, int ny,
                       const double* d_k, const double* d_z, int nz, double depth, float2* spectra) {
	if (nx != 2 * M || ny != NY) return false;
	if constexpr (M * NY > kRealMaxPoints / 2) {
		return false;
	} else {
		// 512 threads where the array takes one CTA per SM (16384 points);
		// 256 below, two CTAs per SM (up to ~70 KB each), so that one CTA's
		// barrier phases overlap the other's work
		constexpr int NT = M * NY >= 16384 ? 512 : 256;
		constexpr int L = 2 * M > NY ? 2 * M : NY;
		const size_t smem = sizeof(float2) * (size_t(M) * RealLd<M, NY>::v + L);
		ARMA_CUDA_TRY(cudaFuncSetAttribute(velocity_real_kernel<M, NY, NT>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		velocity_real_kernel<M, NY, NT><<<ns, NT, smem, c->stream>>>(d_sl, d_k, d_z, nz, depth,
		                                                              spectra);
		return true;
	}
}

template <int M>
bool launch_real_m(Ctx* c, const VelSlice<float>* d_sl, int ns, int nx, int ny, const double* d_k,
                   const double* d_z, int nz, double depth, float2* spectra) {
	return launch_real_shape<M, 16>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_shape<M, 32>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_shape<M, 64>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_shape<M, 128>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_shape<M, 256>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra);
}

// ---------------------------------------------------------------- 2d. real, cluster
// The same solver for slices whose M x NY array (256 KB at 256 x 256) does not
// fit one CTA's shared memory: a cluster of two CTAs, each holding H = M / 2
// pair rows, with the halves exchanged through distributed shared memory.
//   rows:     local NY-point FFTs of each CTA's pair rows
//   columns:  the first radix-2 stage (decimation in frequency) across the
//             halves, y0 = x[i] + x[i+H], y1 = (x[i] - x[i+H]) W_M^i, written
//             to CTA 0 (y0) and CTA 1 (y1) -- each CTA computes the columns of
//             its half of NY, reading and writing both halves -- then local
//             H-point column FFTs: CTA r holds column frequencies 2j + r
//   pairing:  a and -a have the same parity, so every pair is local
//   inverse:  local H-point column FFTs, the radix-2 stage mirrored
//             (x[i] = y0 + W_M^-i y1, x[i+H] = y0 - W_M^-i y1), local row FFTs
// Cluster barriers separate every step that reads the other CTA's memory from
// the writes before and after it.
template <int M, int NY, int NT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NT, 1)
velocity_real2_kernel(const VelSlice<float>* __restrict__ sl, const double* __restrict__ kinfo,
                      const double* __restrict__ zs, int nz, double depth,
                      float2* __restrict__ spectra) {
	namespace cg = cooperative_groups;
	constexpr int NX = 2 * M, H = M / 2, LD = RealLd<H, NY>::v;
	constexpr int L = NX > NY ? NX : NY;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	cg::cluster_group cl = cg::this_cluster();
	const int rank = int(cl.block_rank());
	float2* A = reinterpret_cast<float2*>(smem_raw);  // H rows of LD
	float2* tw = A + H * LD;                           // L
	float2* Ar = cl.map_shared_rank(A, rank ^ 1);      // the other half
	float2* A0 = rank == 0 ? A : Ar;
	float2* A1 = rank == 0 ? Ar : A;
	const int s = blockIdx.x / 2;
	const VelSlice<float> S = sl[s];
	constexpr int n2 = NX * NY;
	for (int j = threadIdx.x; j < L; j += NT) {
		double sn, cs;
		sincospi(2.0 * j / L, &sn, &cs);
		tw[j] = make_float2(float(cs), float(-sn));
	}
	real_input_rows<NY, NT, LD>(S, NX, rank * H, H, A);
	__syncthreads();
	lines_fft<NY, false, NT, false>(A, H, LD, 1, tw, L / NY);  // rows
	cl.sync();
	for (int q = threadIdx.x; q < H * (NY / 2); q += NT) {  // radix-2 across the halves
		const int i = q / (NY / 2), y = rank * (NY / 2) + q % (NY / 2);
		const float2 x0 = A0[i * LD + y], x1 = A1[i * LD + y];
		A0[i * LD + y] = make_float2(x0.x + x1.x, x0.y + x1.y);
		A1[i * LD + y] = cmul_tw<false>(make_float2(x0.x - x1.x, x0.y - x1.y), tw[i * (L / M)]);
	}
	cl.sync();
	lines_fft<H, false, NT, true>(A, NY, 1, LD, tw, L / H);  // columns, local
	__syncthreads();
	float2* spec = spectra ? spectra + (long long)s * M * NY + (long long)rank * H * NY : nullptr;
	if (spec) {
		for (int q = threadIdx.x; q < H * NY; q += NT) spec[q] = A[(q / NY) * LD + q % NY];
		__syncthreads();
	}
	const double wx = 1.0 / kinfo[s * 4 + 0], wy = 1.0 / kinfo[s * 4 + 1];
	const double dkx = wx / (NX - 1), dky = wy / (NY - 1);
	const float inv = float(1.0 / double(M * NY));
	for (int iz = 0; iz < nz; ++iz) {
		if (iz > 0) {
			cl.sync();  // the previous depth's output read both halves
			for (int q = threadIdx.x; q < H * NY; q += NT) A[(q / NY) * LD + q % NY] = spec[q];
			__syncthreads();
		}
		const double z = zs[iz];
		const bool flat = window_flat(NX, NY, dkx, dky, z, depth);
		const float flat_w = float(window_flat_value());
		// pairs {(a, b), (-a, -b)} with a = 2j + rank (local row j)
		for (int q = threadIdx.x; q < H * (NY / 2 + 1); q += NT) {
			const int j = q / (NY / 2 + 1), b = q % (NY / 2 + 1), a = 2 * j + rank;
			if ((b == 0 || b == NY / 2) && a > M / 2) continue;
			const int am = a == 0 ? 0 : M - a, bm = b == 0 ? 0 : NY - b;
			const int jm = (am - rank) / 2;
			const float2 z1 = A[j * LD + b], z2 = A[jm * LD + bm];
			const float2 E = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
			const float2 O = make_float2(0.5f * (z1.y + z2.y), -0.5f * (z1.x - z2.x));
			float2 E2, O2;
			if (flat) {  // S = the constant, D = 0: the same values without the window calls
				E2 = make_float2(flat_w * E.x, flat_w * E.y);
				O2 = make_float2(flat_w * O.x, flat_w * O.y);
			} else {
				const double wa = window_even(a, b, NX, NY, dkx, dky, z, depth);
				const double wb = window_even(a + M, b, NX, NY, dkx, dky, z, depth);
				const float Sv = float(0.5 * (wa + wb)), Dv = float(0.5 * (wa - wb));
				const float2 w = tw[a * (L / NX)];  // W_nx^a
				const float2 wO = cmul_tw<false>(O, w), wE = cmul_tw<true>(E, w);
				E2 = make_float2(Sv * E.x + Dv * wO.x, Sv * E.y + Dv * wO.y);
				O2 = make_float2(Sv * O.x + Dv * wE.x, Sv * O.y + Dv * wE.y);
			}
			A[j * LD + b] = make_float2(E2.x - O2.y, E2.y + O2.x);
			A[jm * LD + bm] = make_float2(E2.x + O2.y, -E2.y + O2.x);
		}
		__syncthreads();
		lines_fft<H, true, NT, true>(A, NY, 1, LD, tw, L / H);  // columns, local
		cl.sync();
		for (int q = threadIdx.x; q < H * (NY / 2); q += NT) {  // radix-2 across the halves
			const int i = q / (NY / 2), y = rank * (NY / 2) + q % (NY / 2);
			const float2 y0 = A0[i * LD + y];
			const float2 y1 = cmul_tw<true>(A1[i * LD + y], tw[i * (L / M)]);
			A0[i * LD + y] = make_float2(y0.x + y1.x, y0.y + y1.y);
			A1[i * LD + y] = make_float2(y0.x - y1.x, y0.y - y1.y);
		}
		cl.sync();
		lines_fft<NY, true, NT, false>(A, H, LD, 1, tw, L / NY);  // rows
		cl.sync();  // the edge fix of the second half reads the first half's last row
		float* out = S.out + (long long)iz * n2;
		auto f = [&](int r, int c) -> double {
			const int pr = r >> 1;
			const float2* src = pr < H ? A0 : A1;
			const float2 v = src[(pr % H) * LD + c];
			return double((r & 1) ? v.y : v.x) * double(inv);
		};
		for (int q = threadIdx.x; q < 2 * H * NY; q += NT) {
			const int x = rank * 2 * H + q / NY, y = q % NY;
			float* o = out + (long long)x * NY + y;
			if (x > 0 && y > 0) {
				const float2 v = A[((x >> 1) - rank * H) * LD + y];
				*o = ((x & 1) ? v.y : v.x) * inv;
			} else {
				*o = float(finish_at(x, y, NX, NY, f));
			}
		}
	}
	cl.sync();  // the other CTA may still read this one's shared memory
}

bool real_path_supported(int nx, int ny) {
	auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
	return pow2(nx) && pow2(ny) && nx >= 32 && nx <= 256 && ny >= 16 && ny <= 256 &&
	       (nx * ny <= kRealMaxPoints || (nx == 256 && ny == 256));
}

bool launch_velocity_real(Ctx* c, const VelSlice<float>* d_sl, int ns, int nx, int ny,
                          const double* d_k, const double* d_z, int nz, double depth,
                          float2* spectra) {
	if (nx == 256 && ny == 256) {  // two CTAs per slice
		constexpr int M = 128, NY = 256, NT = 512, H = M / 2;
		const size_t smem = sizeof(float2) * (size_t(H) * RealLd<H, NY>::v + 256);
		ARMA_CUDA_TRY(cudaFuncSetAttribute(velocity_real2_kernel<M, NY, NT>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		velocity_real2_kernel<M, NY, NT><<<2 * ns, NT, smem, c->stream>>>(d_sl, d_k, d_z, nz, depth,
		                                                                  spectra);
		return true;
	}
	return launch_real_m<16>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_m<32>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_m<64>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra) ||
	       launch_real_m<128>(c, d_sl, ns, nx, ny, d_k, d_z, nz, depth, spectra);
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
	ARMA_CUDA_TRY(copy_async(c, d_sl, slices.data(), sizeof(VelSlice<T>) * ns,
	                              cudaMemcpyHostToDevice, c->stream));
	ARMA_CUDA_TRY(copy_async(c, d_z, z, sizeof(double) * nz, cudaMemcpyHostToDevice, c->stream));
	{
		// pieces per line of the x pass (lines are the ny columns) and the y
		// pass (the nx rows); warps per CTA: the larger axis's units, <= 8;
		// then the other axis's lines are cut further so that its CTAs have a
		// unit for every warp too, where the lines are long enough
		const int b0 = (ny + 31) / 32, b1 = (nx + 31) / 32;
		int p0 = fw_pieces(ny, nx - 2, ns, c->num_sms), p1 = fw_pieces(nx, ny - 2, ns, c->num_sms);
		const int fwarps = std::max(1, std::min(kFwThreads / 32, std::max(b0 * p0, b1 * p1)));
		p0 = std::max(p0, std::min(fw_piece_cap(ny, nx - 2), (fwarps + b0 - 1) / b0));
		p1 = std::max(p1, std::min(fw_piece_cap(nx, ny - 2), (fwarps + b1 - 1) / b1));
		const int nseg = std::max(ny * p0, nx * p1);
		const size_t fw_smem = seg_region_bytes(std::max(nseg, fwarps)) +
		                       sizeof(T) * size_t(fwarps) * fw_tiles<T>() * 32 * kFwTile;
		ARMA_CUDA_TRY(cudaFuncSetAttribute(factor_waves_kernel<T>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(fw_smem)));
		factor_waves_kernel<T><<<2 * ns, 32 * fwarps, fw_smem, c->stream>>>(d_sl, nx, ny, p0, p1, d_k);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
	bool linear_only = true;
	for (const auto& v : slices) linear_only = linear_only && v.mode == 0;
	if (sizeof(T) == sizeof(float) && linear_only && real_path_supported(nx, ny)) {
		float2* spectra =
		    nz > 1 ? static_cast<float2*>(scratch_take(c, sizeof(float2) * (n2 / 2) * ns)) : nullptr;
		ARMA_REQUIRE(launch_velocity_real(c, reinterpret_cast<const VelSlice<float>*>(d_sl), ns, nx,
		                                  ny, d_k, d_z, nz, depth, spectra),
		             ARMA_EINVAL, "velocity solver: no real-input kernel for this slice shape");
		ARMA_CUDA_TRY(cudaGetLastError());
		c->launches += 1;
		return;
	}
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
