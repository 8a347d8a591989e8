// dcmt Mersenne Twister word generation on the device.
//
// The dcmt generator (genrand_mt, called by prng::parallel_mt::operator(),
// reference src/parallel_mt.hh:236) is the MT linear recurrence over a ring of
// nn words followed by tempering.  Written as a sequence of raw words
//     x[j] = x[j-n+m] ^ (y >> 1) ^ (y & 1 ? aaa : 0),
//     y    = (x[j-n] & umask) | (x[j-n+1] & lmask),   j >= n,
// with x[0..n-1] the seeded state (sgenrand_mt), output word w is
// temper(x[n+w]).  Every word of a chunk [j0, j0+n-m) depends only on words
// before j0, so one CTA produces n-m words per barrier step with all
// arithmetic in 32-bit integers; sets with nn = 2 mm run one warp per segment
// with no barrier (mt_generate_half_kernel).
//
// Long streams are cut into segments of J = 2^20 words generated by separate
// CTAs.  The window of nn raw words at the start of segment k is obtained by
// jumping: with g(t) = t^(J 2^l) mod phi(t) (phi the characteristic
// polynomial, mt_jump.cc), the window D positions ahead is the XOR of the
// windows of the raw sequence at the set bits of g.  Segment starts are built
// as a binary tree: level l turns every known start k*2^(l+1) into
// k*2^(l+1) + 2^l.  All of it is bit-identical to the sequential generator.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "internal.h"

namespace armab {

// Defined in mt_jump.cc.
bool mt_jump_tables(const arma_mt_params& prm, int log2_jump, int levels,
                    std::vector<std::vector<int32_t>>* set_bits, int* degree);

namespace {

constexpr int kRingBits = 12;
constexpr int kRing = 1 << kRingBits;  // ring of raw words, >= nn + (nn-mm)
constexpr int kLevels = 16;            // jump tables for J * 2^l, l < 16
constexpr int kJumpThreads = 640;

struct SegJob {
	arma_mt_params p;
	uint32_t seed;
	const uint32_t* state;     // window of nn raw words, or null: seed it
	unsigned long long first;  // output index of the segment's first word
	unsigned long long count;  // words in the segment
	unsigned long long offset; // words before `offset` are not stored
	uint32_t* out;             // out[w - offset] for output index w
};

struct JumpJob {
	arma_mt_params p;
	const uint32_t* src;  // window at position a
	uint32_t* dst;        // window at position a + D
	const int32_t* bits;  // set bits of t^D mod phi
	int nbits;
};

__device__ __forceinline__ uint32_t temper(uint32_t y, const arma_mt_params& p) {
	y ^= y >> p.shift0;
	y ^= (y << p.shiftB) & p.maskB;
	y ^= (y << p.shiftC) & p.maskC;
	y ^= y >> p.shift1;
	return y;
}

__device__ __forceinline__ void seed_state(uint32_t* dst, uint32_t seed, const arma_mt_params& p) {
	// sgenrand_mt: Knuth's 1812433253 initialisation masked by wmask.
	uint32_t s = seed;
	for (int k = 0; k < p.nn; ++k) {
		dst[k] = s & p.wmask;
		s = 1812433253u * (s ^ (s >> 30)) + uint32_t(k + 1);
	}
}

// The block has one thread per word of a chunk of n - m words, rounded up
// to whole warps (up to kGenMaxThreads); longer chunks give each thread W =
// ceil((n - m) / blockDim) words (n - m <= kMaxOwn * kGenMaxThreads covers
// every Mersenne exponent up to 44497 several times over).
constexpr int kGenMaxThreads = 1024;
constexpr int kMaxOwn = 4;

template <int W>
__global__ void __launch_bounds__(kGenMaxThreads)
mt_generate_kernel(const SegJob* __restrict__ jobs) {
	__shared__ uint32_t ring[kRing];
	const SegJob& jb = jobs[blockIdx.x];
	const arma_mt_params p = jb.p;
	const int n = p.nn, m = p.mm;
	const int chunk = n - m;
	const long long count = (long long)jb.count;
	const long long shift = (long long)jb.first - (long long)jb.offset;  // out index - word
	uint32_t* const out = jb.out;
	if (jb.state) {
		for (int k = threadIdx.x; k < n; k += blockDim.x) ring[k] = jb.state[k];
	} else if (threadIdx.x == 0) {
		seed_state(ring, jb.seed, p);
	}
	__syncthreads();
	const uint32_t mask = kRing - 1;
	// Thread t owns words t + i B (B = blockDim, i < W, those < n - m) of every
	// chunk: segment word w = s (n-m) + t + i B at step s, raw word r = n + w
	// at ring position r & mask (positions run modulo 2^32, a multiple of the
	// ring size), so every index is a running register sum.  Each step emits
	// the chunk computed by the step before and computes the next one: raw
	// r + n - m reads raw r (this thread's own word) and raw r - m, r - m + 1,
	// all written in earlier steps.
	auto next_word = [&](uint32_t r) {  // raw word r from raw r - n, r - n + 1, r - n + m
		const uint32_t y = (ring[(r - n) & mask] & p.umask) | (ring[(r - n + 1) & mask] & p.lmask);
		return ring[(r - n + m) & mask] ^ (y >> 1) ^ ((y & 1u) ? p.aaa : 0u);
	};
	uint32_t r[W];
	long long o[W], rem[W];
	bool owner[W];
#pragma unroll
	for (int i = 0; i < W; ++i) {
		const int t = threadIdx.x + i * int(blockDim.x);
		owner[i] = t < chunk;
		r[i] = uint32_t(n + t);  // raw position of this word
		o[i] = shift + t;        // its output index
		rem[i] = count - t;      // words from it to the segment's end
		if (owner[i] && rem[i] > 0) ring[r[i] & mask] = next_word(r[i]);
	}
	__syncthreads();
	const long long steps = (count + chunk - 1) / chunk;
	for (long long st = 0; st < steps; ++st) {
#pragma unroll
		for (int i = 0; i < W; ++i) {
			if (owner[i]) {
				if (rem[i] > 0 && o[i] >= 0) out[o[i]] = temper(ring[r[i] & mask], p);
				if (rem[i] > chunk) ring[(r[i] + chunk) & mask] = next_word(r[i] + chunk);
				r[i] += chunk;
				o[i] += chunk;
				rem[i] -= chunk;
			}
		}
		__syncthreads();
	}
}

// Sets with nn = 2 mm (every committed set of period 2^19937 - 1): with the
// chunk n - m = m, output word w = m s + t (step s, slot t < m) is
//     x[n + w] = x[n + w - m] ^ f(x[w], x[w + 1]),
// where x[n + w - m] is slot t of step s-1, x[w] slot t of step s-2 and
// x[w + 1] slot t+1 of step s-2 (slot 0 of step s-1 when t = m-1): every
// word needs only its own slot's last two values and the next slot's.  One
// warp runs one segment with no barrier: lane l holds slots t = 32 q + l
// (q < kHalfQ) of the last two steps in registers, takes the next slot's
// values by shuffles, and stores each q's 32 words coalesced.  The state
// window (raw words 0 .. n-1) is steps -2 and -1.
constexpr int kHalfQ = 10;     // slots per lane: mm <= 320
constexpr int kHalfWarps = 4;  // warps (segments) per CTA
constexpr int kHalfMaxN = 2 * 32 * kHalfQ;

__host__ __device__ inline bool half_set(const arma_mt_params& p) {
	return p.nn == 2 * p.mm && p.mm <= 32 * kHalfQ;
}

// One step of the warp generator: slots of step s from those of steps s-2 (a)
// and s-1 (b); b0 = slot 0 of step s-1.  M > 0: the compile-time mm (slot
// checks resolved at compile time); M = 0: mm = m at run time.
template <int M>
__device__ __forceinline__ void half_step(const uint32_t* a, const uint32_t* b, uint32_t* nb,
                                          uint32_t b0, int m, int lane, const arma_mt_params& p) {
	const int mm = M > 0 ? M : m;
#pragma unroll
	for (int q = 0; q < kHalfQ; ++q) {
		if (M > 0 && 32 * q >= M) break;
		const int t = 32 * q + lane;
		const uint32_t down = __shfl_down_sync(0xffffffffu, a[q], 1);
		const uint32_t wrap = __shfl_sync(0xffffffffu, q + 1 < kHalfQ ? a[q + 1] : 0u, 0);
		uint32_t a1 = lane < 31 ? down : wrap;
		if ((M == 0 || 32 * q + 31 >= M - 1) && t == mm - 1) a1 = b0;
		const uint32_t y = (a[q] & p.umask) | (a1 & p.lmask);
		nb[q] = b[q] ^ (y >> 1) ^ ((y & 1u) ? p.aaa : 0u);
	}
}

template <int M>
__global__ void __launch_bounds__(32 * kHalfWarps)
mt_generate_half_kernel(const SegJob* __restrict__ jobs, int njobs) {
	__shared__ uint32_t seeded[kHalfWarps][kHalfMaxN];
	const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
	const int g = blockIdx.x * kHalfWarps + wl;
	if (g >= njobs) return;
	const SegJob& jb = jobs[g];
	const arma_mt_params p = jb.p;
	const int m = M > 0 ? M : p.mm;
	const uint32_t* st = jb.state;
	if (!st) {
		if (lane == 0) seed_state(seeded[wl], jb.seed, p);
		__syncwarp();
		st = seeded[wl];
	}
	uint32_t a[kHalfQ], b[kHalfQ];  // slots of steps s-2 and s-1
#pragma unroll
	for (int q = 0; q < kHalfQ; ++q) {
		const int t = 32 * q + lane;
		a[q] = t < m ? st[t] : 0u;
		b[q] = t < m ? st[m + t] : 0u;
	}
	// segment words w < count (<= 2^30) go to out[first - offset + w] when that
	// index is >= 0: base = out + max(first - offset, 0), index w - wmin
	const int count = int(jb.count);
	const long long shift = (long long)jb.first - (long long)jb.offset;
	const int wmin = shift < 0 ? int(-shift) : 0;
	uint32_t* const base = jb.out + (shift > 0 ? shift : 0);
	int w0 = 0;
	if (wmin == 0) {
		// whole steps: every slot < m is stored
		for (; w0 + m <= count; w0 += m) {
			const uint32_t b0 = __shfl_sync(0xffffffffu, b[0], 0);
			uint32_t nb[kHalfQ];
			half_step<M>(a, b, nb, b0, m, lane, p);
			uint32_t* dst = base + w0 + lane;
#pragma unroll
			for (int q = 0; q < kHalfQ; ++q) {
				if (M > 0 && 32 * q >= M) break;
				if ((M > 0 && 32 * q + 32 <= M) || 32 * q + lane < m) dst[32 * q] = temper(nb[q], p);
				a[q] = b[q];
				b[q] = nb[q];
			}
		}
	}
	// the rest: skipped words before the offset, the last partial step
	for (; w0 < count; w0 += m) {
		const uint32_t b0 = __shfl_sync(0xffffffffu, b[0], 0);
		uint32_t nb[kHalfQ];
		half_step<M>(a, b, nb, b0, m, lane, p);
#pragma unroll
		for (int q = 0; q < kHalfQ; ++q) {
			const int t = 32 * q + lane;
			const int w = w0 + t;
			if (t < m && w < count && w >= wmin) base[w - wmin] = temper(nb[q], p);
			a[q] = b[q];
			b[q] = nb[q];
		}
	}
}

// Window of segment 0 of each jumped job: the seeded state, or a copy of the
// job's own window.
__global__ void mt_seed_kernel(const arma_mt_params* __restrict__ ps,
                               const uint32_t* __restrict__ seeds,
                               const uint32_t* const* __restrict__ src, uint32_t* const* dst) {
	const uint32_t* s = src[blockIdx.x];
	if (s) {
		for (int k = threadIdx.x; k < ps[blockIdx.x].nn; k += blockDim.x) dst[blockIdx.x][k] = s[k];
	} else if (threadIdx.x == 0) {
		seed_state(dst[blockIdx.x], seeds[blockIdx.x], ps[blockIdx.x]);
	}
}

// Inverse of temper(): each xor-shift step y ^= (y >> s) (or (y << s) & mask)
// is undone by the fixed-point iteration x <- y ^ (x >> s), which settles s
// more bits per pass.
__device__ __forceinline__ uint32_t undo_right(uint32_t y, int s) {
	uint32_t x = y;
	for (int k = 0; k < 32; k += s) x = y ^ (x >> s);
	return x;
}
__device__ __forceinline__ uint32_t undo_left(uint32_t y, int s, uint32_t mask) {
	uint32_t x = y;
	for (int k = 0; k < 32; k += s) x = y ^ ((x << s) & mask);
	return x;
}
__device__ __forceinline__ uint32_t untemper(uint32_t y, const arma_mt_params& p) {
	y = undo_right(y, p.shift1);
	y = undo_left(y, p.shiftC, p.maskC);
	y = undo_left(y, p.shiftB, p.maskB);
	return undo_right(y, p.shift0);
}

struct WindowJob {
	arma_mt_params p;
	const uint32_t* words;               // tempered words of the last chunk
	unsigned long long n_words;          // words generated for it
	const unsigned long long* attempts;  // polar attempts the chunk consumed
	uint32_t* window;                    // raw window at the next word
	unsigned long long* position;        // running word position (may be null)
};

// The raw window in front of word 4*attempts: untempered copies of the nn
// words before it.  A chunk whose noise ran short reports no attempt count
// (0): the window is left as it was and the chunk is generated again.
__global__ void mt_window_kernel(const WindowJob* __restrict__ jobs) {
	const WindowJob& jb = jobs[blockIdx.x];
	const unsigned long long used = 4ull * *jb.attempts;
	const int n = jb.p.nn;
	if (used < (unsigned long long)n || used > jb.n_words) return;
	for (int k = threadIdx.x; k < n; k += blockDim.x)
		jb.window[k] = untemper(jb.words[used - n + k], jb.p);
	if (threadIdx.x == 0 && jb.position) *jb.position += used;
}

// `parts` CTAs per jump: each computes the raw words y[0 .. p+n-2] from the
// source window in shared memory, then its share of the destination window,
// dst[w] = XOR over the set bits i of y[i + w], with the bit list split among
// several threads per word and the partial XORs combined in shared memory.
// More parts shorten a jump when few jumps run at once.
__global__ void __launch_bounds__(kJumpThreads)
mt_jump_kernel(const JumpJob* __restrict__ jobs, int parts) {
	extern __shared__ uint32_t y[];
	const JumpJob& jb = jobs[blockIdx.x / parts];
	const arma_mt_params p = jb.p;
	const int n = p.nn, m = p.mm, chunk = n - m;
	const int per = (n + parts - 1) / parts;
	const int w0 = (blockIdx.x % parts) * per;
	if (w0 >= n) return;  // uniform over the CTA
	const int cnt = min(n, w0 + per) - w0;
	const int deg = 32 * n - p.rr;
	const int len = deg + n - 1;
	for (int k = threadIdx.x; k < n; k += blockDim.x) y[k] = jb.src[k];
	__syncthreads();
	for (int j0 = n; j0 < len; j0 += chunk) {
		for (int t = threadIdx.x; t < chunk; t += blockDim.x) {
			const int j = j0 + t;
			if (j < len) {
				const uint32_t v = (y[j - n] & p.umask) | (y[j - n + 1] & p.lmask);
				y[j] = y[j - n + m] ^ (v >> 1) ^ ((v & 1u) ? p.aaa : 0u);
			}
		}
		__syncthreads();
	}
	uint32_t* acc = y + len;  // lanes * cnt <= blockDim.x partial XORs
	const int lanes = max(1, int(blockDim.x) / cnt);
	const int wl = threadIdx.x % cnt, lane = threadIdx.x / cnt;
	if (lane < lanes) {
		const int nb = jb.nbits;
		const int span = ((nb + lanes - 1) / lanes + 3) & ~3;  // multiple of 4: aligned int4 loads
		const int b0 = min(nb, lane * span), b1 = min(nb, b0 + span);
		const int w = w0 + wl;
		uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
		int it = b0;
		for (; it + 4 <= b1; it += 4) {
			const int4 b = *reinterpret_cast<const int4*>(jb.bits + it);
			r0 ^= y[b.x + w];
			r1 ^= y[b.y + w];
			r2 ^= y[b.z + w];
			r3 ^= y[b.w + w];
		}
		for (; it < b1; ++it) r0 ^= y[jb.bits[it] + w];
		acc[lane * cnt + wl] = r0 ^ r1 ^ r2 ^ r3;
	}
	__syncthreads();
	for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
		uint32_t r = 0;
		for (int l = 0; l < lanes; ++l) r ^= acc[l * cnt + t];
		jb.dst[w0 + t] = r;
	}
}

std::vector<uint32_t> params_key(const arma_mt_params& p) {
	std::vector<uint32_t> k(sizeof(p) / 4);
	std::memcpy(k.data(), &p, sizeof(p));
	k.back() = 0;  // the `i` field does not affect the stream
	return k;
}

// Jump tables are cached per (device, parameter set, segment length) for the
// life of the process; every context on the device shares them.
struct MtTable {
	bool ok = false;
	std::vector<int32_t*> bits;  // device arrays, one per level
	std::vector<int> nbits;
};
std::mutex g_table_mutex;
std::map<std::vector<uint32_t>, MtTable> g_tables;

const MtTable& jump_table(Ctx* c, const arma_mt_params& p, int log2_seg) {
	auto key = params_key(p);
	key.push_back(uint32_t(c->device));
	key.push_back(uint32_t(log2_seg));
	std::lock_guard<std::mutex> lock(g_table_mutex);
	auto it = g_tables.find(key);
	if (it != g_tables.end()) return it->second;
	MtTable t;
	std::vector<std::vector<int32_t>> bits;
	int deg = 0;
	t.ok = mt_jump_tables(p, log2_seg, kLevels, &bits, &deg);
	if (t.ok) {
		for (auto& b : bits) {
			// pad to a multiple of 4 for vector loads (pads are never read)
			std::vector<int32_t> v = b;
			while (v.size() % 4) v.push_back(0);
			int32_t* d = nullptr;
			ARMA_CUDA_TRY(cudaMalloc(&d, sizeof(int32_t) * std::max<size_t>(v.size(), 4)));
			ARMA_CUDA_TRY(cudaMemcpy(d, v.data(), sizeof(int32_t) * v.size(), cudaMemcpyHostToDevice));
			t.bits.push_back(d);
			t.nbits.push_back(int(b.size()));
		}
	}
	return g_tables.emplace(key, std::move(t)).first->second;
}

}  // namespace

namespace {
// The jump-ahead windows and the generation of a batch of jobs.  prepare:
// only the windows (at every segment start of every job longer than one
// segment), handed back in prepare[q].seg_states; a job that already carries
// seg_states is not jumped again.
void mt_batch(Ctx* c, const std::vector<MtJob>& jobs, int log2_seg, std::vector<MtJob>* prepare) {
	ProfScope prof_(c, "mt");
	ARMA_REQUIRE(log2_seg >= 12 && log2_seg <= 24, ARMA_EINVAL, "bad MT segment length");
	for (const MtJob& j : jobs) {
		ARMA_REQUIRE(!j.state || j.offset == 0, ARMA_EINVAL,
		             "an MT job started from a window has no offset");
		ARMA_REQUIRE(j.p.nn > 1 && j.p.mm > 0 && j.p.mm < j.p.nn && j.p.ww == 32, ARMA_EINVAL,
		             "bad MT parameter set");
		ARMA_REQUIRE(j.p.nn + (j.p.nn - j.p.mm) <= kRing &&
		                 j.p.nn - j.p.mm <= kMaxOwn * kGenMaxThreads,
		             ARMA_EINVAL, "MT state too large for the device generator");
	}
	if (jobs.empty()) return;
	const unsigned long long J = 1ull << log2_seg;
	// segments per job; jobs with more than one segment need jump tables
	std::vector<int> K(jobs.size());
	std::vector<const MtTable*> tab(jobs.size(), nullptr);
	int Kmax = 1;
	size_t nstates = 0;
	std::vector<char> ready(jobs.size(), 0);  // windows precomputed: no jumps here
	std::vector<const uint32_t*> state0(jobs.size(), nullptr);  // per job: K windows of nn words
	for (size_t q = 0; q < jobs.size(); ++q) {
		const unsigned long long total = jobs[q].offset + jobs[q].count;
		ARMA_REQUIRE((total + J - 1) / J <= (1ull << kLevels), ARMA_EINVAL, "MT stream too long");
		K[q] = int(std::max(1ull, (total + J - 1) / J));
		if (jobs[q].seg_states) {
			ARMA_REQUIRE(K[q] > 1, ARMA_EINVAL, "MT job with windows but one segment");
			ready[q] = 1;
			state0[q] = jobs[q].seg_states;
			continue;
		}
		if (K[q] > 1) {
			tab[q] = &jump_table(c, jobs[q].p, log2_seg);
			if (!tab[q]->ok) K[q] = 1;  // not a full-period set: one sequential segment
		}
		if (K[q] > 1) nstates += size_t(K[q]) * jobs[q].p.nn;
		Kmax = std::max(Kmax, K[q]);
	}
	if (nstates) {
		uint32_t* states = static_cast<uint32_t*>(scratch_take(c, sizeof(uint32_t) * nstates));
		size_t off = 0;
		std::vector<arma_mt_params> ps;
		std::vector<uint32_t> seeds;
		std::vector<const uint32_t*> src;
		std::vector<uint32_t*> dst;
		for (size_t q = 0; q < jobs.size(); ++q) {
			if (K[q] <= 1 || ready[q]) continue;
			state0[q] = states + off;
			off += size_t(K[q]) * jobs[q].p.nn;
			ps.push_back(jobs[q].p);
			seeds.push_back(jobs[q].seed);
			src.push_back(jobs[q].state);
			dst.push_back(states + (state0[q] - states));
		}
		auto* d_ps = static_cast<arma_mt_params*>(scratch_take(c, sizeof(arma_mt_params) * ps.size()));
		auto* d_seeds = static_cast<uint32_t*>(scratch_take(c, sizeof(uint32_t) * seeds.size()));
		auto* d_src = static_cast<const uint32_t**>(scratch_take(c, sizeof(uint32_t*) * src.size()));
		auto* d_dst = static_cast<uint32_t**>(scratch_take(c, sizeof(uint32_t*) * dst.size()));
		ARMA_CUDA_TRY(copy_async(c, d_ps, ps.data(), sizeof(arma_mt_params) * ps.size(),
		                              cudaMemcpyHostToDevice, c->stream));
		ARMA_CUDA_TRY(copy_async(c, d_seeds, seeds.data(), sizeof(uint32_t) * seeds.size(),
		                              cudaMemcpyHostToDevice, c->stream));
		ARMA_CUDA_TRY(copy_async(c, d_src, src.data(), sizeof(uint32_t*) * src.size(),
		                              cudaMemcpyHostToDevice, c->stream));
		ARMA_CUDA_TRY(copy_async(c, d_dst, dst.data(), sizeof(uint32_t*) * dst.size(),
		                              cudaMemcpyHostToDevice, c->stream));
		mt_seed_kernel<<<int(ps.size()), 32, 0, c->stream>>>(d_ps, d_seeds, d_src, d_dst);
		c->launches += 1;
		// binary tree of jumps, widest stride first
		int levels = 0;
		while ((1 << levels) < Kmax) ++levels;
		size_t smem = 0;
		for (size_t q = 0; q < jobs.size(); ++q)
			if (K[q] > 1 && !ready[q])
				smem = std::max(smem, sizeof(uint32_t) * size_t(32 * jobs[q].p.nn - jobs[q].p.rr +
				                                                jobs[q].p.nn + kJumpThreads));
		ARMA_CUDA_TRY(cudaFuncSetAttribute(mt_jump_kernel,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		for (int lv = levels - 1; lv >= 0; --lv) {
			std::vector<JumpJob> jj;
			const int step = 1 << lv;
			for (size_t q = 0; q < jobs.size(); ++q) {
				if (K[q] <= 1 || ready[q]) continue;
				const int nn = jobs[q].p.nn;
				uint32_t* w = states + (state0[q] - states);
				for (int base = 0; base + step < K[q]; base += 2 * step)
					jj.push_back(JumpJob{jobs[q].p, w + size_t(base) * nn, w + size_t(base + step) * nn,
					                     tab[q]->bits[lv], tab[q]->nbits[lv]});
			}
			if (jj.empty()) continue;
			auto* d_jj = static_cast<JumpJob*>(scratch_take(c, sizeof(JumpJob) * jj.size()));
			ARMA_CUDA_TRY(copy_async(c, d_jj, jj.data(), sizeof(JumpJob) * jj.size(),
			                              cudaMemcpyHostToDevice, c->stream));
			// few jumps at this level: split each over several CTAs
			int parts = int(std::min<size_t>(8, std::max<size_t>(1, (2 * size_t(c->num_sms) +
			                                                         jj.size() - 1) / jj.size())));
			for (const JumpJob& j : jj)  // every CTA's share must fit one word per thread
				parts = std::max(parts, (j.p.nn + kJumpThreads - 1) / kJumpThreads);
			mt_jump_kernel<<<int(jj.size()) * parts, kJumpThreads, smem, c->stream>>>(d_jj, parts);
			ARMA_CUDA_TRY(cudaGetLastError());
			c->launches += 1;
		}
	}
	if (prepare) {
		for (size_t q = 0; q < jobs.size(); ++q)
			if (K[q] > 1) (*prepare)[q].seg_states = state0[q];
		return;
	}
	// generation: one CTA per segment
	std::vector<SegJob> seg;
	for (size_t q = 0; q < jobs.size(); ++q) {
		const unsigned long long total = jobs[q].offset + jobs[q].count;
		for (int k = 0; k < K[q]; ++k) {
			const unsigned long long first = (unsigned long long)k * J;
			if (K[q] > 1 && first + J <= jobs[q].offset) continue;  // entirely skipped
			SegJob s;
			s.p = jobs[q].p;
			s.seed = jobs[q].seed;
			s.state = K[q] > 1 ? state0[q] + size_t(k) * jobs[q].p.nn : jobs[q].state;
			s.first = first;
			s.count = K[q] > 1 ? std::min(J, total - first) : total;
			s.offset = jobs[q].offset;
			s.out = jobs[q].out;
			seg.push_back(s);
		}
	}
	// segments of nn = 2 mm sets: one warp each (32-bit word indices); the
	// rest: one CTA each
	auto by_warp = [](const SegJob& j) {
		return half_set(j.p) && j.count < (1ull << 30) && j.offset < (1ull << 30) &&
		       j.first < (1ull << 40);
	};
	std::stable_partition(seg.begin(), seg.end(), by_warp);
	const int nhalf = int(std::count_if(seg.begin(), seg.end(), by_warp));
	auto* d_seg = static_cast<SegJob*>(scratch_take(c, sizeof(SegJob) * seg.size()));
	ARMA_CUDA_TRY(copy_async(c, d_seg, seg.data(), sizeof(SegJob) * seg.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	if (nhalf > 0) {
		// mm = 312 (the sets of period 2^19937 - 1) compiled in; others at run time
		bool all312 = true;
		for (int k = 0; k < nhalf; ++k) all312 = all312 && seg[k].p.mm == 312;
		const int hgrid = (nhalf + kHalfWarps - 1) / kHalfWarps;
		if (all312)
			mt_generate_half_kernel<312><<<hgrid, 32 * kHalfWarps, 0, c->stream>>>(d_seg, nhalf);
		else
			mt_generate_half_kernel<0><<<hgrid, 32 * kHalfWarps, 0, c->stream>>>(d_seg, nhalf);
		ARMA_CUDA_TRY(cudaGetLastError());
		c->launches += 1;
	}
	const int grid = int(seg.size()) - nhalf;
	if (grid > 0) {
		int chunk = 1;  // the largest chunk of the rest
		for (size_t k = size_t(nhalf); k < seg.size(); ++k)
			chunk = std::max(chunk, seg[k].p.nn - seg[k].p.mm);
		const int threads = std::min(kGenMaxThreads, (chunk + 31) / 32 * 32);
		const int own = (chunk + threads - 1) / threads;
		const SegJob* rest = d_seg + nhalf;
		switch (own) {
			case 1: mt_generate_kernel<1><<<grid, threads, 0, c->stream>>>(rest); break;
			case 2: mt_generate_kernel<2><<<grid, threads, 0, c->stream>>>(rest); break;
			case 3: mt_generate_kernel<3><<<grid, threads, 0, c->stream>>>(rest); break;
			default: mt_generate_kernel<4><<<grid, threads, 0, c->stream>>>(rest); break;
		}
		ARMA_CUDA_TRY(cudaGetLastError());
		c->launches += 1;
	}
}

}  // namespace

void launch_mt_generate_batch(Ctx* c, const std::vector<MtJob>& jobs, int log2_seg) {
	mt_batch(c, jobs, log2_seg, nullptr);
}

void launch_mt_prepare(Ctx* c, std::vector<MtJob>& jobs, int log2_seg) {
	mt_batch(c, jobs, log2_seg, &jobs);
}

void launch_mt_window_update(Ctx* c, const std::vector<MtWindowSpec>& specs) {
	if (specs.empty()) return;
	ProfScope prof_(c, "mt");
	std::vector<WindowJob> jobs(specs.size());
	for (size_t k = 0; k < specs.size(); ++k)
		jobs[k] = WindowJob{specs[k].p, specs[k].words, specs[k].n_words, specs[k].attempts,
		                    specs[k].window, specs[k].position};
	auto* d_jobs = static_cast<WindowJob*>(scratch_take(c, sizeof(WindowJob) * jobs.size()));
	ARMA_CUDA_TRY(copy_async(c, d_jobs, jobs.data(), sizeof(WindowJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	mt_window_kernel<<<int(jobs.size()), 256, 0, c->stream>>>(d_jobs);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

void launch_mt_generate(Ctx* c, const arma_mt_params& p, uint32_t seed,
                        uint64_t offset, uint64_t n, uint32_t* d_out) {
	if (n == 0) return;
	launch_mt_generate_batch(c, {MtJob{p, seed, offset, n, d_out}});
	// the job tables live in scratch and pageable host vectors: finish first
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
}

}  // namespace armab
