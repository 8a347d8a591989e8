// FP32 compensated AR filter: a persistent tile wavefront over a batch of
// independent surfaces.
//
// The filter (reference src/generator/ar_model_surf.cc:5-36) is
//     zeta(t,x,y) = eps(t,x,y) + sum_{(k,i,j) != 0} phi(k,i,j) zeta(t-k,x-i,y-j)
// with zeta = 0 outside the array.  Because phi(0,i,j) != 0, every point
// depends on earlier points of its own time slice as well as on the previous
// pt-1 slices.  The work is split into spatial tiles of TX x TY points; one
// CTA owns one tile of one surface for all t and walks the slices in order.
// For slice t its four compute warps
//   1. accumulate the terms on slices t-1 .. t-pt+1 (90% of the work for a
//      10^3 model) from a shared-memory ring that holds those slices for the
//      tile plus its west/north halo,
//   2.-3. meanwhile a fifth warp publishes slice t-1, clears the ring slot of
//      slice t, waits for the three neighbour tiles (x-1, y-1, both) to
//      publish slice t (a per-tile counter in global memory; bounded spin)
//      and loads slice t of the halo; then the compute warps add the
//      current-slice terms that reach into the halo (the in-tile part of the
//      current slice is held at zero),
//   4. solve the remaining in-tile recursion zeta = S + A0 zeta exactly as a
//      quarter-plane convolution zeta = H * S, where H is the impulse response
//      of 1 / (1 - A0(z1,z2)) on the tile (precomputed in FP64),
//   5. store the slice to the ring and to global memory; the fifth warp
//      publishes it (release store after a fence) off the compute warps'
//      critical path.
// The coefficients are carried as hi + lo float pairs (rounding phi to one
// float perturbs a high-gain recursion far more than FP32 summation does):
// each (k,i) row of taps feeds two FP32 FMA chains over one register window,
// continued across the rows of one k plane, and the plane totals are combined
// with Kahan compensation (per row, the compensation cost 7 % more time for
// 0.2-1.2e-6 less RMS error).  H is applied in plain FP32, one FMA chain per
// output over up to three rows of H (up to 96 taps), the at most six chain
// totals of an output Kahan-added: it acts once per slice on the current
// slice alone, and its rounding changes the surface by far less than phi's (a
// lo part for H moved the RMS error by under 1e-7 at 18 % of the filter's
// time; Kahan-adding every row of H instead of every three rows, by 4e-8 at
// 5 %).  Tiles are handed out through a global ticket
// counter in dependency order, so a CTA only ever waits on tiles that are
// already owned by running CTAs.
#include <algorithm>
#include <climits>
#include <mutex>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr int TX = 16;            // tile rows (x)
constexpr int TY = 32;            // tile columns (y)
constexpr int R = 8;              // outputs per thread along y
constexpr int STRIPS = TY / R;    // threads per tile row
constexpr int GROUP = TX * STRIPS; // threads covering the tile once
constexpr int NCOMP = 2 * GROUP;   // compute threads: two groups split the tap rows
constexpr int NTHREADS = NCOMP + 32; // plus the halo / publication warp
// named barriers (0 is __syncthreads)
constexpr int BAR_HALO = 1;        // halo warp -> compute: slot t cleared, halo of t loaded
constexpr int BAR_COMP = 2;        // compute threads among themselves
constexpr int BAR_DONE = 3;        // compute -> halo warp: slice t stored
constexpr int LH = 12;            // left (y) halo columns held in the ring
constexpr int W = LH + TY;        // ring row width (floats)
constexpr int SPAD = TY + 8;      // zero padding left of each S row
constexpr int SW = SPAD + TY + 4; // S row width (padded against bank conflicts)
constexpr int MAXO = 13;          // max order per axis supported (py <= LH+1)
constexpr int HS = TY + 4;        // H row stride in shared memory (bank spread)
constexpr int HCH = 3;            // rows of H per H work unit
constexpr int HPAIR = 51;         // H work units per strip pair: sum_x ceil((x+1)/HCH)
constexpr int HUNITS = 2 * HPAIR; // H work units per tile slice (<= NCOMP)
constexpr int PS = 2 * R + 4;     // partial record stride (bank spread)
static_assert(TX == 16 && TY == 4 * R && HUNITS <= NCOMP, "H work-unit table assumes 16 x 4R tiles");
constexpr int kMaxTapRows = MAXO * (TX + 1);  // (k, i) tap rows per model: pt * px
constexpr long long kSpinLimit = 1ll << 24;

struct Task {
	int nt, nx, ny, pt, px, py;
	int t0;  // slices [0, t0) are history: read, never written
	int given_tx;  // tile rows [0, given_tx) are given (an x-strip's upper band): read, never written
	int tiles_x, tiles_y;
	int ticket_base;
	float* zeta;
	const float* phi;     // hi part, pt*px*py
	const float* phi_lo;  // lo part: phi - hi, pt*px*py
	const float* h;       // intra-slice response, TX*TY
	int* flags;
};

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
	const float y = v - c;
	const float t = s + y;
	c = (t - s) - y;
	s = t;
}

__device__ __forceinline__ void cp_async16(float* dst_smem, const float* src) {
	const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst_smem));
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void bar_sync(int id, int n) {
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void bar_arrive(int id, int n) {
	asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
	asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p) {
	int v;
	asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
	asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until every non-null flag is >= need; the three acquire loads of a
// poll are issued together so one L2 round trip covers them.  seen[] holds the
// values this thread's earlier acquire loads returned: a neighbour that is
// already known to be at or past `need` is not polled again (that load's
// acquire already ordered its slices before this thread's later loads), so a
// tile whose neighbours run ahead pays no round trip.  Gives up after
// kSpinLimit polls (or when another CTA already gave up) and reports
// DEV_TIMEOUT; returns false then.
__device__ bool wait_flags(const int* f0, const int* f1, const int* f2, int need, int* seen,
                           int* err) {
	if (seen[0] >= need && seen[1] >= need && seen[2] >= need) return true;
	for (long long it = 0; it < kSpinLimit; ++it) {
		const int a = f0 ? ld_acquire(f0) : need;
		const int b = f1 ? ld_acquire(f1) : need;
		const int c = f2 ? ld_acquire(f2) : need;
		seen[0] = f0 ? a : INT_MAX;
		seen[1] = f1 ? b : INT_MAX;
		seen[2] = f2 ? c : INT_MAX;
		if (a >= need && b >= need && c >= need) return true;
		if ((it & 63) == 63 && *((volatile int*)err) != DEV_OK) return false;
		__nanosleep(64);
	}
	atomicExch(err, DEV_TIMEOUT);
	return false;
}

// zeta = H * S over the quarter plane of one tile, cut into work units of
// equal cost.  Row x of the output needs the x+1 rows dx = 0..x of H, each a
// causal 1-D convolution along y; the four 8-column strips of a row cost 1, 2,
// 3 and 4 blocks of R x R taps (the first block of each a triangle), so the
// strips are paired (3, 0) and (2, 1): either pair costs two triangles and
// three full blocks per row of H.  A unit is one strip pair of one output row
// over at most HCH consecutive rows of H; units are numbered pair-major, then
// by row, then by dx chunk, so row x's units start at HPAIR * pair +
// h_rowbase(x).  Unit u writes its partial (strip X in slots 0..R-1, strip Y
// in R..2R-1), one plain FP32 FMA chain per output, to part[u * PS ..]; the
// partials of an output are Kahan-added afterwards.  Lanes of one warp work
// on different rows of H at once: H rows are HS floats apart in shared memory
// so that their 16-byte loads fall in different banks.  The unit is inlined
// into every tap-count instantiation of run_tile: as a call, the registers
// the caller keeps across it spilled, and the filter ran 7 % slower.
__device__ __forceinline__ int h_rowbase(int x) {
	// sum over x' < x of ceil((x'+1) / HCH), for HCH = 3
	const int q = x / 3, r = x % 3;
	return x + 3 * q * (q - 1) / 2 + r * q;
}

__device__ __forceinline__ void load_row(float* d, const float* s, int n4) {
#pragma unroll 4
	for (int q = 0; q < n4; ++q) {
		const float4 v = reinterpret_cast<const float4*>(s)[q];
		d[4 * q] = v.x;
		d[4 * q + 1] = v.y;
		d[4 * q + 2] = v.z;
		d[4 * q + 3] = v.w;
	}
}

// acc[r] += sum_dd hv[dd] src[R + r - dd]: one full R x R block of taps
__device__ __forceinline__ void h_block(float* acc, const float* src, const float* hrow) {
	float w[2 * R], hv[R];
	load_row(w, src, 2 * R / 4);
	load_row(hv, hrow, R / 4);
#pragma unroll
	for (int r = 0; r < R; ++r) {
#pragma unroll
		for (int dd = 0; dd < R; ++dd) acc[r] = fmaf(hv[dd], w[R + r - dd], acc[r]);
	}
}

__device__ __forceinline__ void h_unit(const float* ss, const float* sh, int u, float* part) {
	const int pair = u >= HPAIR ? 1 : 0;
	const int v = u - pair * HPAIR;
	int x = 0;
	while (x + 1 < TX && h_rowbase(x + 1) <= v) ++x;
	const int dx0 = HCH * (v - h_rowbase(x));
	const int dx1 = min(dx0 + HCH, x + 1);
	const int yx = pair ? 2 * R : 3 * R;  // first column of strip X
	const int yy = pair ? R : 0;          // first column of strip Y
	const int w3 = pair ? 0 : 2 * R;      // sources of the third block
	// one FMA chain per output over the unit's rows of H
	float pX[R], pY[R];
#pragma unroll
	for (int r = 0; r < R; ++r) { pX[r] = 0.0f; pY[r] = 0.0f; }
	for (int dx = dx0; dx < dx1; ++dx) {
		const float* srow = ss + (x - dx) * SW + SPAD;
		const float* hrow = sh + dx * HS;
		float wt[R], hv[R];
		// triangle of strip X: its block dy0 = yx reaches sources srow[0 .. r]
		load_row(wt, srow, R / 4);
		load_row(hv, hrow + yx, R / 4);
#pragma unroll
		for (int r = 0; r < R; ++r) {
#pragma unroll
			for (int dd = 0; dd <= r; ++dd) pX[r] = fmaf(hv[dd], wt[r - dd], pX[r]);
		}
		// strip X's blocks dy0 = yx - R and yx - 2R
		h_block(pX, srow, hrow + yx - R);
		h_block(pX, srow + R, hrow + yx - 2 * R);
		// third block: strip 3's dy0 = 0 (pair 0) or strip 1's dy0 = 0 (pair 1)
		float q[R];
#pragma unroll
		for (int r = 0; r < R; ++r) q[r] = pair ? pY[r] : pX[r];
		h_block(q, srow + w3, hrow);
#pragma unroll
		for (int r = 0; r < R; ++r) {
			pX[r] = pair ? pX[r] : q[r];
			pY[r] = pair ? q[r] : pY[r];
		}
		// triangle of strip Y
		load_row(hv, hrow + yy, R / 4);
#pragma unroll
		for (int r = 0; r < R; ++r) {
#pragma unroll
			for (int dd = 0; dd <= r; ++dd) pY[r] = fmaf(hv[dd], wt[r - dd], pY[r]);
		}
	}
	float* out = part + u * PS;
#pragma unroll
	for (int q4 = 0; q4 < R / 4; ++q4) {
		reinterpret_cast<float4*>(out)[q4] =
		    make_float4(pX[4 * q4], pX[4 * q4 + 1], pX[4 * q4 + 2], pX[4 * q4 + 3]);
		reinterpret_cast<float4*>(out + R)[q4] =
		    make_float4(pY[4 * q4], pY[4 * q4 + 1], pY[4 * q4 + 2], pY[4 * q4 + 3]);
	}
}

template <int PY>
__device__ void run_tile(const Task& tk, int bx, int by, float* smem, unsigned char* s_lo,
                         int* err) {
	const int tid = threadIdx.x;
	if (bx < tk.given_tx) {
		// a given tile (the band above an x-strip, holding the upper strip's
		// finished values): published as complete for every slice at once
		if (tid == 0) st_release(tk.flags + bx * tk.tiles_y + by, tk.nt);
		return;
	}
	const int grp = tid / GROUP;                 // 0 or 1: halves of the tap rows
	const int lt = tid % GROUP;
	const int xl = lt / STRIPS;                  // tile-local row
	const int yl0 = (lt % STRIPS) * R;           // tile-local first column
	const int pt = tk.pt, px = tk.px;
	const int hx = px - 1;
	const int rows = TX + hx;
	const int slot_sz = rows * W;
	constexpr int PYP = (PY + 3) & ~3;           // padded tap row
	const int x0 = bx * TX, y0 = by * TY;
	const long long sst = (long long)tk.nx * tk.ny;

	float* ring = smem;                          // pt slots
	float* sphi = ring + pt * slot_sz;           // pt*px*PYP (hi)
	float* slo = sphi + pt * px * PYP;           // pt*px*PYP (lo)
	float* sh = slo + pt * px * PYP;             // TX*HS
	float* ss = sh + TX * HS;                    // TX*SW
	float* part = ss + TX * SW;                  // HUNITS*PS: H-unit partials
	float* comb = part;                          // GROUP*R: group 1 partials (before H)

	// stage coefficients (rows padded with zeros), H, zero the ring and S pads
	for (int q = tid; q < pt * px * PYP; q += NTHREADS) {
		const int j = q % PYP, ki = q / PYP;
		sphi[q] = j < PY ? tk.phi[ki * PY + j] : 0.0f;
		slo[q] = j < PY ? tk.phi_lo[ki * PY + j] : 0.0f;
	}
	// rows whose lo parts are all zero skip their second FMA chain
	for (int ki = tid; ki < pt * px; ki += NTHREADS) {
		bool nz = false;
		for (int j = 0; j < PY; ++j) nz = nz || tk.phi_lo[ki * PY + j] != 0.0f;
		s_lo[ki] = nz ? 1 : 0;
	}
	for (int q = tid; q < TX * TY; q += NTHREADS) sh[(q / TY) * HS + q % TY] = tk.h[q];
	for (int q = tid; q < pt * slot_sz; q += NTHREADS) ring[q] = 0.0f;
	for (int q = tid; q < TX * SW; q += NTHREADS) ss[q] = 0.0f;
	__syncthreads();
	// history slices (a stream's previous chunk): the whole ring slot, tile
	// and halo, straight from global memory (zero outside the surface)
	for (int tt = max(0, tk.t0 - pt + 1); tt < tk.t0; ++tt) {
		float* slot = ring + (tt % pt) * slot_sz;
		const float* zs = tk.zeta + tt * sst;
		for (int q = tid; q < slot_sz; q += NTHREADS) {
			const int x = x0 - hx + q / W, y = y0 - LH + q % W;
			if (x >= 0 && x < tk.nx && y >= 0 && y < tk.ny) slot[q] = __ldcg(zs + (long long)x * tk.ny + y);
		}
	}
	__syncthreads();

	__shared__ int s_ok;
	if (tid >= NCOMP) {
		// The halo / publication warp.  For slice t it waits until the compute
		// threads have stored slice t-1 (which also ends their use of slot t's
		// previous contents), publishes slice t-1, clears slot t, waits for the
		// three neighbour tiles to publish slice t and loads slice t's halo,
		// while the compute threads accumulate the previous slices' terms.
		const int lane = tid - NCOMP;
		// 16-byte halo chunks need 16-byte aligned rows in global memory
		const bool vec_ok = (tk.ny % 4 == 0) &&
		                    ((reinterpret_cast<uintptr_t>(tk.zeta) & 15) == 0) && ((sst % 4) == 0);
		const int* fW = (bx > 0) ? tk.flags + (bx - 1) * tk.tiles_y + by : nullptr;
		const int* fN = (by > 0) ? tk.flags + bx * tk.tiles_y + by - 1 : nullptr;
		const int* fNW = (bx > 0 && by > 0) ? tk.flags + (bx - 1) * tk.tiles_y + by - 1 : nullptr;
		int* own_flag = tk.flags + bx * tk.tiles_y + by;
		int seen[3] = {-1, -1, -1};
		for (int t = tk.t0; t < tk.nt; ++t) {
			// the release store orders the compute threads' stores of slice
			// t-1 (made visible to this thread by the barrier) before the flag
			if (t > tk.t0) {
				bar_sync(BAR_DONE, NTHREADS);
				if (lane == 0) st_release(own_flag, t);
			}
			float* cur = ring + (t % pt) * slot_sz;
			const float* zt = tk.zeta + t * sst;
			for (int q = lane; q < slot_sz; q += 32) cur[q] = 0.0f;
			__syncwarp();
			int ok = 1;
			if (lane == 0) ok = wait_flags(fW, fN, fNW, t + 1, seen, err) ? 1 : 0;
			ok = __shfl_sync(0xffffffffu, ok, 0);
			if (ok) {
				// rows above the tile (all columns) and the left columns of the
				// tile rows, in 16-byte chunks copied with L2-only asynchronous
				// copies (scalar loads at ragged edges)
				const int top = hx * (W / 4);
				const int nch = top + TX * (LH / 4);
				for (int q = lane; q < nch; q += 32) {
					int rr, c4;
					if (q < top) {
						rr = q / (W / 4);
						c4 = q % (W / 4);
					} else {
						rr = hx + (q - top) / (LH / 4);
						c4 = (q - top) % (LH / 4);
					}
					const int x = x0 - hx + rr, y = y0 - LH + 4 * c4;
					if (x < 0 || x >= tk.nx) continue;  // stays zero
					float* dst = cur + rr * W + 4 * c4;
					const float* src = zt + (long long)x * tk.ny + y;
					if (vec_ok && y >= 0 && y + 4 <= tk.ny) {
						cp_async16(dst, src);
					} else {
						for (int e = 0; e < 4; ++e)
							if (y + e >= 0 && y + e < tk.ny) dst[e] = __ldcg(src + e);
					}
				}
				cp_async_wait_all();
			}
			if (lane == 0) s_ok = ok;
			bar_arrive(BAR_HALO, NTHREADS);
			if (!ok) return;
		}
		if (tk.nt > tk.t0) {
			bar_sync(BAR_DONE, NTHREADS);
			if (lane == 0) st_release(own_flag, tk.nt);
		}
		return;
	}

	const int gx = x0 + xl;

	for (int t = tk.t0; t < tk.nt; ++t) {
		float* cur = ring + (t % pt) * slot_sz;
		float* zt = tk.zeta + t * sst;
		// group 0 starts from the noise of its strip (own tile: written by an
		// earlier kernel), group 1 from zero
		float s[R], c[R];
#pragma unroll
		for (int r = 0; r < R; ++r) {
			const int gy = y0 + yl0 + r;
			s[r] = (grp == 0 && gx < tk.nx && gy < tk.ny) ? zt[(long long)gx * tk.ny + gy] : 0.0f;
			c[r] = 0.0f;
		}
		// One (k, i) row of taps at a time, rows alternating between the two
		// groups: the hi and lo coefficient parts are applied as two FP32 FMA
		// chains over the same register window, each chain running across the
		// rows of the k plane; the plane total is Kahan-added to the running
		// sum.
		auto accumulate_rows = [&](const float* slot, int k) {
			const float* prow = sphi + (k * px) * PYP;
			const float* lrow = slo + (k * px) * PYP;
			float pk[R], qk[R];
#pragma unroll
			for (int r = 0; r < R; ++r) { pk[r] = 0.0f; qk[r] = 0.0f; }
			for (int i = (k * px + grp) & 1; i < px; i += 2) {
				const float* zr = slot + (xl + hx - i) * W + yl0;
				float win[R + LH];
#pragma unroll
				for (int q = 0; q < (R + LH) / 4; ++q) {
					const float4 v = reinterpret_cast<const float4*>(zr)[q];
					win[4 * q] = v.x;
					win[4 * q + 1] = v.y;
					win[4 * q + 2] = v.z;
					win[4 * q + 3] = v.w;
				}
				float ph[PYP];
#pragma unroll
				for (int q = 0; q < PYP / 4; ++q) {
					const float4 v = reinterpret_cast<const float4*>(prow + i * PYP)[q];
					ph[4 * q] = v.x;
					ph[4 * q + 1] = v.y;
					ph[4 * q + 2] = v.z;
					ph[4 * q + 3] = v.w;
				}
				if (s_lo[k * px + i]) {  // warp-uniform: every thread handles this row
					float pl[PYP];
#pragma unroll
					for (int q = 0; q < PYP / 4; ++q) {
						const float4 u = reinterpret_cast<const float4*>(lrow + i * PYP)[q];
						pl[4 * q] = u.x;
						pl[4 * q + 1] = u.y;
						pl[4 * q + 2] = u.z;
						pl[4 * q + 3] = u.w;
					}
#pragma unroll
					for (int r = 0; r < R; ++r) {
#pragma unroll
						for (int j = 0; j < PY; ++j) {
							pk[r] = fmaf(ph[j], win[LH + r - j], pk[r]);
							qk[r] = fmaf(pl[j], win[LH + r - j], qk[r]);
						}
					}
				} else {
#pragma unroll
					for (int r = 0; r < R; ++r) {
#pragma unroll
						for (int j = 0; j < PY; ++j) pk[r] = fmaf(ph[j], win[LH + r - j], pk[r]);
					}
				}
			}
#pragma unroll
			for (int r = 0; r < R; ++r) kahan_add(s[r], c[r], pk[r] + qk[r]);
		};

		// 1. previous slices (the halo warp meanwhile prepares slot t)
		for (int k = 1; k < pt && k <= t; ++k) accumulate_rows(ring + ((t - k) % pt) * slot_sz, k);

		// 2./3. slot t cleared, neighbours' slice t published, halo loaded
		bar_sync(BAR_HALO, NTHREADS);
		if (!s_ok) return;
		accumulate_rows(cur, 0);

		// 4. S = noise + all terms outside the unknown in-tile part
		if (grp == 1) {
#pragma unroll
			for (int r = 0; r < R; ++r) comb[lt * R + r] = s[r] - c[r];
		}
		bar_sync(BAR_COMP, NCOMP);
		if (grp == 0) {
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int gy = y0 + yl0 + r;
				const bool valid = gx < tk.nx && gy < tk.ny;
				ss[xl * SW + SPAD + yl0 + r] = valid ? (s[r] + (comb[lt * R + r] - c[r])) : 0.0f;
			}
		}
		bar_sync(BAR_COMP, NCOMP);

		//    zeta = H * S over the quarter plane of the tile, in work units
		if (tid < HUNITS) h_unit(ss, sh, tid, part);

		// 5. sum each output's unit partials (Kahan, in dx order), store the
		//    solved slice; the halo warp publishes it
		bar_sync(BAR_COMP, NCOMP);
		{
			// this thread's outputs: row ox, columns oy0 .. oy0+3
			const int ox = tid / (2 * STRIPS);
			const int ostrip = (tid / 2) % STRIPS;
			const int oy0 = ostrip * R + (tid % 2) * 4;
			const int opart = (ostrip == 0 || ostrip == 3 ? 0 : HPAIR) + h_rowbase(ox);
			const int oslot = (ostrip >= 2 ? 0 : R) + (tid % 2) * 4;
			const int ogx = x0 + ox;
			float a[4], ac[4];
#pragma unroll
			for (int e = 0; e < 4; ++e) { a[e] = 0.0f; ac[e] = 0.0f; }
			const int nch = ox / HCH + 1;
			for (int ch = 0; ch < nch; ++ch) {
				const float4 v = *reinterpret_cast<const float4*>(part + (opart + ch) * PS + oslot);
				kahan_add(a[0], ac[0], v.x);
				kahan_add(a[1], ac[1], v.y);
				kahan_add(a[2], ac[2], v.z);
				kahan_add(a[3], ac[3], v.w);
			}
			float* own = cur + hx * W + LH + ox * W + oy0;
#pragma unroll
			for (int e = 0; e < 4; ++e) {
				const float v = a[e] - ac[e];
				own[e] = v;
				const int gy = y0 + oy0 + e;
				if (ogx < tk.nx && gy < tk.ny) zt[(long long)ogx * tk.ny + gy] = v;
			}
		}
		bar_sync(BAR_COMP, NCOMP);  // slice t in the ring for every compute thread
		bar_arrive(BAR_DONE, NTHREADS);
	}
}

// One launch for the whole batch: each ticket's surface selects the
// instantiation for its tap count py (warp-uniform switch).
__global__ void __launch_bounds__(NTHREADS, 3)
ar32c_kernel(const Task* __restrict__ tasks, int ntasks, int total_tickets,
             int* __restrict__ ticket_counter, int* __restrict__ err) {
	extern __shared__ __align__(16) float smem[];
	__shared__ int s_ticket;
	__shared__ unsigned char s_lo[kMaxTapRows];  // per (k, i) tap row: lo part present
	for (;;) {
		if (threadIdx.x == 0) s_ticket = atomicAdd(ticket_counter, 1);
		__syncthreads();
		const int ticket = s_ticket;
		__syncthreads();
		if (ticket >= total_tickets) return;
		if (*((volatile int*)err) != DEV_OK) return;
		// locate the surface owning this ticket
		int lo = 0, hi = ntasks - 1;
		while (lo < hi) {
			const int mid = (lo + hi + 1) / 2;
			if (tasks[mid].ticket_base <= ticket) lo = mid; else hi = mid - 1;
		}
		const Task tk = tasks[lo];
		const int local = ticket - tk.ticket_base;
		const int bx = local / tk.tiles_y, by = local % tk.tiles_y;
		switch (tk.py) {
#define ARMA_PY_CASE(N) case N: run_tile<N>(tk, bx, by, smem, s_lo, err); break;
			ARMA_PY_CASE(1) ARMA_PY_CASE(2) ARMA_PY_CASE(3) ARMA_PY_CASE(4) ARMA_PY_CASE(5)
			ARMA_PY_CASE(6) ARMA_PY_CASE(7) ARMA_PY_CASE(8) ARMA_PY_CASE(9) ARMA_PY_CASE(10)
			ARMA_PY_CASE(11) ARMA_PY_CASE(12) ARMA_PY_CASE(13)
#undef ARMA_PY_CASE
			default: break;
		}
		__syncthreads();
	}
}

size_t smem_bytes(int pt, int px, int py) {
	const int rows = TX + px - 1;
	const int pyp = (py + 3) & ~3;
	return sizeof(float) * (size_t(pt) * rows * W + 2 * size_t(pt) * px * pyp + TX * HS + TX * SW +
	                        std::max(GROUP * R, HUNITS * PS));
}

// The filter's neighbour wait on a tile flag that nothing publishes: it runs
// out after kSpinLimit polls and sets the error word (the failure path of
// every bounded wait, exercised on purpose).
__global__ void wait_selftest_kernel(const int* flag, int* err) {
	int seen[3] = {-1, -1, -1};
	if (threadIdx.x == 0) wait_flags(flag, nullptr, nullptr, 1, seen, err);
}

}  // namespace

void launch_wait_selftest(Ctx* c) {
	int* flag = static_cast<int*>(scratch_take(c, sizeof(int)));
	ARMA_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), c->stream));
	wait_selftest_kernel<<<1, 32, 0, c->stream>>>(flag, c->d_err);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

int ar32c_tile_x() { return TX; }
int ar32c_tile_y() { return TY; }
int ar32c_max_tap_rows() { return kMaxTapRows; }

void launch_ar32c(Ctx* c, const std::vector<Ar32Surface>& surfaces, int tx, int ty, int) {
	ARMA_REQUIRE(tx == TX && ty == TY, ARMA_EINVAL, "unsupported AR tile shape");
	std::vector<int> order(surfaces.size());
	size_t smem = 0;
	for (size_t k = 0; k < surfaces.size(); ++k) {
		const Ar32Surface& s = surfaces[k];
		ARMA_REQUIRE(s.px <= TX + 1 && s.py <= MAXO && s.pt >= 1 && s.px >= 1 && s.py >= 1 &&
		                 s.pt * s.px <= kMaxTapRows,
		             ARMA_ENOTSUP, "AR order not supported by the FP32 tile kernel");
		order[k] = int(k);
		smem = std::max(smem, smem_bytes(s.pt, s.px, s.py));
	}
	// longest dependency chains first: a surface's wavefront needs about
	// nt + tiles_x + tiles_y slice steps, each proportional to pt*px*py
	auto chain = [&](const Ar32Surface& s) {
		return double(s.nt + s.tiles_x + s.tiles_y) * s.pt * s.px * s.py;
	};
	std::sort(order.begin(), order.end(),
	          [&](int a, int b) { return chain(surfaces[a]) > chain(surfaces[b]); });
	size_t nflags = 0;
	for (const auto& s : surfaces) nflags += size_t(s.tiles_x) * s.tiles_y;
	int* flags = static_cast<int*>(scratch_take(c, sizeof(int) * nflags));
	ARMA_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * nflags, c->stream));
	std::vector<Task> tasks;
	int total = 0;
	size_t foff = 0;
	for (int k : order) {
		const Ar32Surface& s = surfaces[k];
		Task t;
		t.nt = s.nt; t.nx = s.nx; t.ny = s.ny;
		t.pt = s.pt; t.px = s.px; t.py = s.py;
		t.t0 = s.t0;
		t.given_tx = s.given_tx;
		t.tiles_x = s.tiles_x; t.tiles_y = s.tiles_y;
		t.ticket_base = total;
		t.zeta = s.zeta; t.phi = s.phi; t.phi_lo = s.phi_lo; t.h = s.h;
		t.flags = flags + foff;
		foff += size_t(s.tiles_x) * s.tiles_y;
		total += s.tiles_x * s.tiles_y;
		tasks.push_back(t);
	}
	Task* d_tasks = static_cast<Task*>(scratch_take(c, sizeof(Task) * tasks.size()));
	int* d_ticket = static_cast<int*>(scratch_take(c, sizeof(int)));
	ARMA_CUDA_TRY(copy_async(c, d_tasks, tasks.data(), sizeof(Task) * tasks.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	ARMA_CUDA_TRY(cudaMemsetAsync(d_ticket, 0, sizeof(int), c->stream));
	ARMA_CUDA_TRY(cudaFuncSetAttribute(ar32c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                   int(smem)));
	int per_sm = 0;
	ARMA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ar32c_kernel, NTHREADS,
	                                                            smem));
	ARMA_REQUIRE(per_sm > 0, ARMA_EINVAL, "AR tile does not fit in shared memory");
	if (c->tuning.ar_ctas_per_sm > 0) per_sm = std::min(per_sm, c->tuning.ar_ctas_per_sm);
	const int grid = std::min(total, per_sm * c->num_sms);
	ProfScope prof_(c, "ar32c");
	ar32c_kernel<<<grid, NTHREADS, smem, c->stream>>>(d_tasks, int(tasks.size()), total, d_ticket,
	                                                  c->d_err);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

}  // namespace armab

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the point where they filter a
// surface: code that runs inside another framework's memory pool and must not
// make stray cudaMalloc calls, latency-bound serving loops that forbid
// allocation (and its implicit synchronisation) on the request path, and
// plugins loaded into processes whose allocator owns the whole device.  This
// entry point runs the same FP32 filter kernel on one surface with every
// piece of scratch it needs (the tile task, the ticket counter, the error
// word, the per-tile publication counters and the hi/lo coefficient and
// intra-slice-response tables) in one file-scope __device__ array of
// kStaticScratchBytes (64 KiB), which every GPU that loads this library holds
// until the process exits.
//
//   * Limits: at most kStaticMaxTiles (8192) tiles of 16 x 32 points per time
//     slice and at most kStaticMaxTaps (2048) AR coefficients; larger
//     requests are rejected with ARMA_EINVAL.  Orders follow the FP32 filter's
//     own limits (at most 16 per axis, px <= 17, py <= 13, pt * px <= 221)
//     and answer ARMA_ENOTSUP beyond them, as arma_ar_filter does.
//   * The coefficient tables are the ones the context path builds
//     (ar32_coefficients), so the result is bit-identical to
//     arma_ar_filter(..., ARMA_FP32C, ...) on the same input.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, under a lock).
//   * Every call reads the device error word back and synchronises the
//     stream before it returns, and stages its tables from host stack
//     memory, so it cannot run under stream capture: a capturing stream is
//     refused with ARMA_EINVAL.
//   * Every call reuses the same array and leaves the last call's contents in
//     it; each call clears the counters it relies on.  Calls whose work
//     overlaps on the GPU (other streams or threads) race on the array and
//     must be serialised by the caller.
//   * It calls no cudaMalloc, cudaFree or allocating library routine.
namespace armab {
namespace {

constexpr size_t kStaticScratchBytes = 64 * 1024;
constexpr int kStaticMaxTiles = 8192;
constexpr int kStaticMaxTaps = 2048;
// byte offsets inside the array; the coefficient block is hi[P], lo[P], H[TX*TY]
constexpr size_t kOffTask = 0;
constexpr size_t kOffTicket = 256;
constexpr size_t kOffErr = 260;
constexpr size_t kOffFlags = 512;
constexpr size_t kOffCoef = kOffFlags + sizeof(int) * kStaticMaxTiles;
constexpr size_t kMaxCoefFloats = 2 * size_t(kStaticMaxTaps) + size_t(TX) * TY;
constexpr size_t kStaticEnd = kOffCoef + sizeof(float) * kMaxCoefFloats;
static_assert(kStaticEnd <= kStaticScratchBytes, "static scratch layout overflows");
static_assert(sizeof(Task) <= kOffTicket, "task record overflows its slot");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_lock;
unsigned char* g_static_addr[kMaxDevices] = {nullptr};

// The array's device address on the current device (looked up once per
// device); nullptr when the lookup fails.
unsigned char* static_scratch(int dev) {
	std::lock_guard<std::mutex> lk(g_static_lock);
	if (!g_static_addr[dev]) {
		void* p = nullptr;
		if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess) return nullptr;
		g_static_addr[dev] = static_cast<unsigned char*>(p);
	}
	return g_static_addr[dev];
}

}  // namespace
}  // namespace armab

extern "C" int arma_ar_filter_fp32c_noalloc(void* stream, const double* phi, const int order[3],
                                            const int shape[3], float* d_zeta) {
	using namespace armab;
	// A failed runtime call leaves the runtime's last-error state set; clear it
	// so that neither this call's launch check nor a later one reads it.
	auto fail = [](int code, const char* msg) {
		(void)cudaGetLastError();
		set_error(msg);
		return code;
	};
	(void)cudaGetLastError();
	if (!phi || !order || !shape || !d_zeta) return fail(ARMA_EINVAL, "null argument");
	if (shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0)
		return fail(ARMA_EINVAL, "Bad \"out_grid\": dimensions must be positive");
	if (order[0] < 1 || order[1] < 1 || order[2] < 1 || order[0] > 16 || order[1] > 16 ||
	    order[2] > 16)
		return fail(ARMA_ENOTSUP, "AR order above 16 per dimension is not supported on the device");
	if (order[1] > TX + 1 || order[2] > MAXO || order[0] * order[1] > kMaxTapRows)
		return fail(ARMA_ENOTSUP, "AR order not supported by the FP32 tile kernel");
	const int P = order[0] * order[1] * order[2];
	if (P > kStaticMaxTaps)
		return fail(ARMA_EINVAL, "allocation-free AR filter: more than 2048 coefficients");
	const int tiles_x = (shape[1] + TX - 1) / TX, tiles_y = (shape[2] + TY - 1) / TY;
	if ((long long)tiles_x * tiles_y > kStaticMaxTiles)
		return fail(ARMA_EINVAL,
		            "allocation-free AR filter: slice needs more than 8192 tiles of 16x32 points");
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(st, &cap) != cudaSuccess)
		return fail(ARMA_ECUDA, "cudaStreamIsCapturing failed");
	if (cap != cudaStreamCaptureStatusNone)
		return fail(ARMA_EINVAL,
		            "allocation-free AR filter: the stream is capturing (the call synchronises)");
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
		return fail(ARMA_ECUDA, "cudaGetDevice failed");
	const size_t smem = smem_bytes(order[0], order[1], order[2]);
	int smem_optin = 0;
	if (cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
	    cudaSuccess)
		return fail(ARMA_ECUDA, "shared-memory limit query failed");
	if (smem > size_t(smem_optin))
		return fail(ARMA_ENOTSUP, "AR order needs more shared memory than the device has");
	unsigned char* base = static_scratch(dev);
	if (!base) return fail(ARMA_ECUDA, "cudaGetSymbolAddress of the static scratch failed");
	if (cudaFuncSetAttribute(ar32c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                         int(smem)) != cudaSuccess)
		return fail(ARMA_ECUDA, "cudaFuncSetAttribute failed");
	float* d_coef = reinterpret_cast<float*>(base + kOffCoef);
	// the context path's tables (hi/lo split, lo-row selection, H), built into
	// host stack memory: 2P + TX*TY <= kMaxCoefFloats floats
	float cbuf[kMaxCoefFloats];
	const size_t ncoef = ar32_coefficient_count(order);
	ar32_coefficients(phi, order, cbuf);
	Task t;
	t.nt = shape[0]; t.nx = shape[1]; t.ny = shape[2];
	t.pt = order[0]; t.px = order[1]; t.py = order[2];
	t.t0 = 0;
	t.given_tx = 0;
	t.tiles_x = tiles_x; t.tiles_y = tiles_y;
	t.ticket_base = 0;
	t.zeta = d_zeta;
	t.phi = d_coef;
	t.phi_lo = d_coef + P;
	t.h = d_coef + 2 * P;
	t.flags = reinterpret_cast<int*>(base + kOffFlags);
	int* d_ticket = reinterpret_cast<int*>(base + kOffTicket);
	int* d_err = reinterpret_cast<int*>(base + kOffErr);
	const int ntiles = tiles_x * tiles_y;
	int per_sm = 0, sms = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ar32c_kernel, NTHREADS, smem) !=
	        cudaSuccess ||
	    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
		return fail(ARMA_ECUDA, "occupancy query failed");
	if (per_sm <= 0) return fail(ARMA_ENOTSUP, "AR tile does not fit in shared memory");
	const int grid = std::min(ntiles, per_sm * sms);
	if (cudaMemcpyAsync(base + kOffTask, &t, sizeof(t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
	    cudaMemcpyAsync(d_coef, cbuf, sizeof(float) * ncoef, cudaMemcpyHostToDevice, st) !=
	        cudaSuccess ||
	    cudaMemsetAsync(base + kOffTicket, 0, 8, st) != cudaSuccess ||
	    cudaMemsetAsync(t.flags, 0, sizeof(int) * ntiles, st) != cudaSuccess) {
		(void)cudaStreamSynchronize(st);  // the staged host buffers are on this stack
		return fail(ARMA_ECUDA, "staging the allocation-free AR filter failed");
	}
	ar32c_kernel<<<grid, NTHREADS, smem, st>>>(reinterpret_cast<const Task*>(base + kOffTask), 1,
	                                           ntiles, d_ticket, d_err);
	const bool launched = cudaGetLastError() == cudaSuccess;
	int herr = 0;
	const bool copied =
	    cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess;
	// wait in every case: the stream still reads this stack's buffers
	const bool synced = cudaStreamSynchronize(st) == cudaSuccess;
	if (!launched) return fail(ARMA_ECUDA, "AR kernel launch failed");
	if (!copied || !synced) return fail(ARMA_ECUDA, "AR kernel failed");
	if (herr == DEV_TIMEOUT)
		return fail(ARMA_ETIMEDOUT, "a bounded device wait gave up (tile dependency not met)");
	if (herr != DEV_OK) return fail(ARMA_ECUDA, "device-side check failed");
	return ARMA_OK;
}
