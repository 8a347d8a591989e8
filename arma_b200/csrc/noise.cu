// Normal white noise from a dcmt word stream, bit-compatible with libstdc++'s
// std::normal_distribution<double> driven by a 32-bit engine.
//
// The reference fills the surface with `dist(mt)` in C order
// (src/white_noise.hh:41-56, src/generator/basic_arma_model.cc:36-48).
// libstdc++ draws each uniform with generate_canonical<double,53> from two
// 32-bit words, u = round53(w0 + w1*2^32) / 2^64, and runs the Marsaglia
// polar method: x = 2u1-1, y = 2u2-1, r2 = x*x + y*y, rejected when r2 > 1 or
// r2 == 0; an accepted attempt yields y*m and then (cached) x*m with
// m = sqrt(-2 log(r2) / r2), each scaled by stddev and offset by the mean 0.
// Every attempt consumes exactly four words, so attempt a reads words
// 4a..4a+3: acceptance is evaluated for all attempts in parallel and a prefix
// sum over accepted attempts gives each pair its output slot.  All arithmetic
// that decides acceptance uses explicitly rounded IEEE double operations (no
// FMA contraction), so the accepted set is exactly the CPU's; log() may
// differ from glibc's by an ulp, so values agree to ~1e-16 relative.
#include "internal.h"

namespace armab {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 4;                      // attempts per thread
constexpr int kPerBlock = kThreads * kPerThread;   // attempts per block

struct Attempt {
	double x, y, r2;
	bool ok;
};

// 2u - 1 for u = generate_canonical(w0, w1) = round53(w0 + w1 2^32) 2^-64,
// clamped to nextafter(1, 0): s = RN(w1 2^32 + w0) is the 64-bit integer
// rounded to double once (as the sum of the two exact doubles is), 2u = s 2^-63
// exactly, and fma(s, 2^-63, -1) rounds 2u - 1 once, as RN(RN(2u) - 1) does.
// u reaches 1 exactly when s = 2^64; it is then nextafter(1, 0) and
// 2u - 1 = 1 - 2^-52.
__device__ __forceinline__ double polar_coordinate(uint32_t w0, uint32_t w1) {
	const double s = __ull2double_rn((static_cast<unsigned long long>(w1) << 32) | w0);
	if (s >= 0x1p64) return 0x1.ffffffffffffep-1;
	return __fma_rn(s, 0x1p-63, -1.0);
}

__device__ __forceinline__ Attempt attempt(uint4 w) {
	Attempt a;
	a.x = polar_coordinate(w.x, w.y);
	a.y = polar_coordinate(w.z, w.w);
	a.r2 = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
	a.ok = !(a.r2 > 1.0 || a.r2 == 0.0);
	return a;
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
	__shared__ int warp_sums[kThreads / 32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = v;
	for (int o = 1; o < 32; o <<= 1) {
		const int t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += t;
	}
	if (lane == 31) warp_sums[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		int s = (lane < kThreads / 32) ? warp_sums[lane] : 0;
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += t;
		}
		if (lane < kThreads / 32) warp_sums[lane] = s;
	}
	__syncthreads();
	const int base = warp ? warp_sums[warp - 1] : 0;
	*total = warp_sums[kThreads / 32 - 1];
	__syncthreads();
	return base + incl - v;
}

__global__ void __launch_bounds__(kThreads)
noise_count_kernel(const uint4* __restrict__ words, unsigned long long n_attempts,
                   int* __restrict__ block_counts) {
	const unsigned long long a0 = (unsigned long long)blockIdx.x * kPerBlock +
	                              (unsigned long long)threadIdx.x * kPerThread;
	int cnt = 0;
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		const unsigned long long a = a0 + k;
		if (a < n_attempts) cnt += attempt(words[a]).ok ? 1 : 0;
	}
	int total;
	block_exclusive_scan(cnt, &total);
	if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

// Exclusive scan of per-block counts (one CTA, sequential over chunks).
__global__ void __launch_bounds__(kThreads)
scan_counts_kernel(const int* __restrict__ counts, int nblocks,
                   long long* __restrict__ offsets, long long* __restrict__ total) {
	__shared__ long long carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (int base = 0; base < nblocks; base += kThreads) {
		const int i = base + threadIdx.x;
		const int v = i < nblocks ? counts[i] : 0;
		int tot;
		const int ex = block_exclusive_scan(v, &tot);
		if (i < nblocks) offsets[i] = carry + ex;
		__syncthreads();
		if (threadIdx.x == 0) carry += tot;
		__syncthreads();
	}
	if (threadIdx.x == 0) *total = carry;
}

template <class T>
__global__ void __launch_bounds__(kThreads)
noise_scatter_kernel(const uint4* __restrict__ words, unsigned long long n_attempts,
                     const long long* __restrict__ block_offsets, double stddev,
                     unsigned long long n, T* __restrict__ out) {
	const unsigned long long a0 = (unsigned long long)blockIdx.x * kPerBlock +
	                              (unsigned long long)threadIdx.x * kPerThread;
	Attempt at[kPerThread];
	int cnt = 0;
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		const unsigned long long a = a0 + k;
		if (a < n_attempts) {
			at[k] = attempt(words[a]);
		} else {
			at[k].ok = false;
		}
		cnt += at[k].ok ? 1 : 0;
	}
	int total;
	long long rank = block_offsets[blockIdx.x] + block_exclusive_scan(cnt, &total);
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		if (!at[k].ok) continue;
		const unsigned long long i0 = 2ull * (unsigned long long)rank;
		if (i0 < n) {
			const double m = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(at[k].r2)), at[k].r2));
			const double v0 = __dadd_rn(__dmul_rn(__dmul_rn(at[k].y, m), stddev), 0.0);
			out[i0] = T(v0);
			if (i0 + 1 < n) {
				const double v1 = __dadd_rn(__dmul_rn(__dmul_rn(at[k].x, m), stddev), 0.0);
				out[i0 + 1] = T(v1);
			}
		}
		++rank;
	}
}

}  // namespace

void enqueue_white_noise(Ctx* c, const uint32_t* d_words, uint64_t n_words,
                         double stddev, uint64_t n, int precision, void* d_out,
                         long long* d_pairs) {
	ProfScope prof_(c, "noise");
	const uint64_t n_attempts = n_words / 4;
	const uint64_t nblocks64 = (n_attempts + kPerBlock - 1) / kPerBlock;
	ARMA_REQUIRE(nblocks64 < (1u << 30), ARMA_EINVAL, "white noise too large");
	const int nblocks = int(nblocks64 ? nblocks64 : 1);
	int* counts = static_cast<int*>(scratch_take(c, sizeof(int) * nblocks));
	long long* offsets = static_cast<long long*>(scratch_take(c, sizeof(long long) * nblocks));
	const uint4* w = reinterpret_cast<const uint4*>(d_words);
	noise_count_kernel<<<nblocks, kThreads, 0, c->stream>>>(w, n_attempts, counts);
	scan_counts_kernel<<<1, kThreads, 0, c->stream>>>(counts, nblocks, offsets, d_pairs);
	if (precision == ARMA_FP64)
		noise_scatter_kernel<double><<<nblocks, kThreads, 0, c->stream>>>(
		    w, n_attempts, offsets, stddev, n, static_cast<double*>(d_out));
	else
		noise_scatter_kernel<float><<<nblocks, kThreads, 0, c->stream>>>(
		    w, n_attempts, offsets, stddev, n, static_cast<float*>(d_out));
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 3;
}

bool launch_white_noise(Ctx* c, const uint32_t* d_words, uint64_t n_words,
                        double stddev, uint64_t n, int precision, void* d_out) {
	long long* total = static_cast<long long*>(scratch_take(c, sizeof(long long)));
	enqueue_white_noise(c, d_words, n_words, stddev, n, precision, d_out, total);
	long long h_total = 0;
	ARMA_CUDA_TRY(copy_async(c, &h_total, total, sizeof(h_total), cudaMemcpyDeviceToHost, c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	return uint64_t(h_total) * 2 >= n;
}

}  // namespace armab

// ---------------------------------------------------------------------------
// Batched form: every surface's polar transform in one launch over tiles of
// kTile attempts.  Tiles take tickets in the order their blocks start (an
// atomic counter); ticket g belongs to the surface whose [block_base, next
// block_base) range holds it (binary search over the surface table).
//
// Within a tile, attempt k kThreads + t (k < kRounds) belongs to thread t, so
// every load and every round's stores are coalesced; its rank among the tile's
// accepted attempts comes from the round's warp ballots and a scan of the
// per-(round, warp) counts.  A pass over the tile counts its accepted attempts
// (keeping one bit per attempt), and a second pass re-reads the words (from
// L1 / L2) and writes the pairs.
//
// The tile's first output slot is the number of pairs the surface's earlier
// tiles accept, found by a decoupled look-back: each tile publishes its own
// count (flag 1) as soon as it has it and its inclusive prefix (flag 2) once it
// knows it, and warp 0 sums the published counts of up to kWindow predecessors
// at a time back to the nearest inclusive prefix (the surface's first tile
// publishes its inclusive prefix at once).  Every tile a ticket holder waits
// for took its ticket earlier, so it is resident and publishes without
// waiting; each wait is still bounded, after which the context's error word is
// set to DEV_TIMEOUT and the tile goes on.
namespace armab {
namespace {

constexpr int kRounds = 16;
constexpr int kTile = kThreads * kRounds;   // attempts per tile
constexpr int kWarps = kThreads / 32;
constexpr int kLook = 4;                    // predecessors per lane per look-back step
constexpr int kWindow = 32 * kLook;
constexpr long long kLookbackSpins = 1ll << 22;

struct NoiseJob {
	const uint4* words;
	unsigned long long n_attempts;
	unsigned long long n;
	double stddev;
	void* out;
	unsigned long long* attempts;
	int block_base;
	int nblocks;
};

__device__ __forceinline__ int find_job(const NoiseJob* jobs, int njobs, int g) {
	int lo = 0, hi = njobs - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) / 2;
		if (jobs[mid].block_base <= g) lo = mid; else hi = mid - 1;
	}
	return lo;
}

// status word: count or inclusive prefix << 2 | flag (1 count, 2 prefix)
__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
	unsigned long long v;
	asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_status(unsigned long long* p, unsigned long long v) {
	asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Sum of the surface's pairs before tile g (warp 0, every lane returns it).
__device__ long long look_back(const unsigned long long* status, int g, int base, int* err) {
	const int lane = threadIdx.x & 31;
	long long excl = 0;
	for (int end = g - 1;; end -= kWindow) {
		// lane l reads predecessors end - l kLook - j, j < kLook (nearest first)
		unsigned long long v[kLook];
		bool gave_up = false;
#pragma unroll
		for (int j = 0; j < kLook; ++j) {
			const int q = end - lane * kLook - j;
			v[j] = 2ull;  // before the surface's first tile: an inclusive prefix of 0
			if (q >= base) {
				v[j] = ld_status(status + q);
				for (long long it = 0; (v[j] & 3ull) == 0ull && !gave_up; ++it) {
					if (it >= kLookbackSpins) gave_up = true;
					__nanosleep(32);
					v[j] = ld_status(status + q);
				}
			}
		}
		if (__any_sync(0xffffffffu, gave_up)) {
			if (lane == 0) atomicExch(err, DEV_TIMEOUT);
			return excl;
		}
		// the nearest inclusive prefix: lane first, then j
		int near = kLook;
#pragma unroll
		for (int j = kLook - 1; j >= 0; --j)
			if ((v[j] & 3ull) == 2ull) near = j;
		const unsigned has = __ballot_sync(0xffffffffu, near < kLook);
		const int stop = has ? __ffs(has) - 1 : 32;  // lane holding it
		long long part = 0;
#pragma unroll
		for (int j = 0; j < kLook; ++j)
			if (lane < stop || (lane == stop && j <= near)) part += (long long)(v[j] >> 2);
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
		excl += part;
		if (has) return excl;
	}
}

template <class T>
__global__ void __launch_bounds__(kThreads)
noise_batch_kernel(const NoiseJob* __restrict__ jobs, int njobs,
                   unsigned long long* __restrict__ status, unsigned int* __restrict__ ticket,
                   long long* __restrict__ pairs, int* __restrict__ err) {
	extern __shared__ __align__(16) unsigned char noise_smem[];  // 2 kTile values of T
	__shared__ int s_g, s_total;
	__shared__ long long s_excl;
	__shared__ int s_cnt[kRounds * kWarps];  // per (round, warp); then their exclusive scan
	if (threadIdx.x == 0) s_g = int(atomicAdd(ticket, 1u));
	__syncthreads();
	const int g = s_g;
	const int sj = find_job(jobs, njobs, g);
	const NoiseJob& jb = jobs[sj];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const unsigned long long tile0 = (unsigned long long)(g - jb.block_base) * kTile;
	const uint4* words = jb.words;
	const unsigned long long na = jb.n_attempts;

	// pass 1: acceptance bits and per-(round, warp) counts
	unsigned okbits = 0;
#pragma unroll 4
	for (int k = 0; k < kRounds; ++k) {
		const unsigned long long a = tile0 + (unsigned long long)k * kThreads + threadIdx.x;
		const bool ok = a < na && attempt(words[a]).ok;
		okbits |= ok ? (1u << k) : 0u;
		const unsigned bal = __ballot_sync(0xffffffffu, ok);
		if (lane == 0) s_cnt[k * kWarps + warp] = __popc(bal);
	}
	__syncthreads();
	if (warp == 0) {
		// exclusive scan of the kRounds * kWarps counts in (round, warp) order
		constexpr int kPerLane = kRounds * kWarps / 32;
		int c[kPerLane], sum = 0;
#pragma unroll
		for (int j = 0; j < kPerLane; ++j) {
			c[j] = s_cnt[lane * kPerLane + j];
			sum += c[j];
		}
		int incl = sum;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o) incl += t;
		}
		int run = incl - sum;
#pragma unroll
		for (int j = 0; j < kPerLane; ++j) {
			s_cnt[lane * kPerLane + j] = run;
			run += c[j];
		}
		const int total = __shfl_sync(0xffffffffu, incl, 31);
		// the tile's own count goes out at once: successors look past it
		if (lane == 0) {
			s_total = total;
			st_status(status + g, ((unsigned long long)total << 2) |
			                          (g == jb.block_base ? 2ull : 1ull));
		}
	}
	__syncthreads();

	// pass 2: the accepted attempts' pairs, in tile order, into shared memory
	// (before the tile's first output slot is known, so that the FP64
	// arithmetic runs while the predecessors publish theirs)
	T* buf = reinterpret_cast<T*>(noise_smem);
	const unsigned below = (1u << lane) - 1u;
#pragma unroll 2
	for (int k = 0; k < kRounds; ++k) {
		const bool ok = (okbits >> k) & 1u;
		const unsigned bal = __ballot_sync(0xffffffffu, ok);
		if (!ok) continue;
		const unsigned long long a = tile0 + (unsigned long long)k * kThreads + threadIdx.x;
		const Attempt at = attempt(words[a]);
		const int lr = s_cnt[k * kWarps + warp] + __popc(bal & below);
		const double m = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(at.r2)), at.r2));
		buf[2 * lr] = T(__dadd_rn(__dmul_rn(__dmul_rn(at.y, m), jb.stddev), 0.0));
		buf[2 * lr + 1] = T(__dadd_rn(__dmul_rn(__dmul_rn(at.x, m), jb.stddev), 0.0));
	}
	// the first output slot: the surface's pairs before this tile
	if (warp == 0) {
		const int total = s_total;
		long long excl = 0;
		if (g != jb.block_base) {
			excl = look_back(status, g, jb.block_base, err);
			if (lane == 0) st_status(status + g, ((unsigned long long)(excl + total) << 2) | 2ull);
		}
		if (lane == 0) {
			s_excl = excl;
			if (g - jb.block_base + 1 == jb.nblocks) pairs[sj] = excl + total;
		}
	}
	__syncthreads();

	// the tile's values to their slots (coalesced), up to the surface's n
	T* out = static_cast<T*>(jb.out);
	const long long excl = s_excl;
	const unsigned long long o0 = 2ull * (unsigned long long)excl;
	const int nv = 2 * s_total;
	for (int q = threadIdx.x; q < nv; q += kThreads)
		if (o0 + q < jb.n) out[o0 + q] = buf[q];
	// a chunk that continues a stream: the attempts consumed up to the pair
	// that ends at value n
	if (jb.attempts && jb.n >= o0 + 2 && jb.n <= o0 + nv) {
		const long long want = (long long)(jb.n - o0) / 2 - 1;  // local rank of that pair
#pragma unroll 2
		for (int k = 0; k < kRounds; ++k) {
			const bool ok = (okbits >> k) & 1u;
			const unsigned bal = __ballot_sync(0xffffffffu, ok);
			if (ok && s_cnt[k * kWarps + warp] + __popc(bal & below) == want)
				*jb.attempts = tile0 + (unsigned long long)k * kThreads + threadIdx.x + 1;
		}
	}
}

}  // namespace

void enqueue_white_noise_batch(Ctx* c, const std::vector<NoiseSpec>& specs, int precision,
                               long long* d_pairs) {
	ProfScope prof_(c, "noise");
	std::vector<NoiseJob> jobs(specs.size());
	long long total_tiles = 0;
	for (size_t k = 0; k < specs.size(); ++k) {
		const uint64_t na = specs[k].n_words / 4;
		const long long nb = (long long)std::max<uint64_t>(1, (na + kTile - 1) / kTile);
		ARMA_REQUIRE(!specs[k].attempts || specs[k].n % 2 == 0, ARMA_EINVAL,
		             "a noise chunk that continues a stream needs an even count");
		jobs[k] = NoiseJob{reinterpret_cast<const uint4*>(specs[k].words), na, specs[k].n,
		                   specs[k].stddev, specs[k].out, specs[k].attempts, int(total_tiles),
		                   int(nb)};
		total_tiles += nb;
	}
	ARMA_REQUIRE(total_tiles < (1ll << 31), ARMA_EINVAL, "white noise batch too large");
	if (jobs.empty()) return;
	auto* d_jobs = static_cast<NoiseJob*>(scratch_take(c, sizeof(NoiseJob) * jobs.size()));
	// the ticket counter, then one status word per tile, zeroed together
	const size_t sync_bytes = sizeof(unsigned long long) * (size_t(total_tiles) + 1);
	auto* sync = static_cast<unsigned long long*>(scratch_take(c, sync_bytes));
	ARMA_CUDA_TRY(cudaMemsetAsync(sync, 0, sync_bytes, c->stream));
	ARMA_CUDA_TRY(copy_async(c, d_jobs, jobs.data(), sizeof(NoiseJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	const int nj = int(jobs.size());
	auto* ticket = reinterpret_cast<unsigned int*>(sync);
	if (precision == ARMA_FP64) {
		const size_t smem = 2 * sizeof(double) * kTile;
		ARMA_CUDA_TRY(cudaFuncSetAttribute(noise_batch_kernel<double>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		noise_batch_kernel<double><<<int(total_tiles), kThreads, smem, c->stream>>>(
		    d_jobs, nj, sync + 1, ticket, d_pairs, c->d_err);
	} else {
		noise_batch_kernel<float><<<int(total_tiles), kThreads, 2 * sizeof(float) * kTile,
		                            c->stream>>>(d_jobs, nj, sync + 1, ticket, d_pairs, c->d_err);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

}  // namespace armab
