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

__device__ __forceinline__ double canonical(uint32_t w0, uint32_t w1) {
	double s = __dadd_rn(double(w0), __dmul_rn(double(w1), 4294967296.0));
	double r = __dmul_rn(s, 5.42101086242752217003726400434970855712890625e-20);  // 2^-64
	if (r >= 1.0) r = 0.99999999999999988897769753748434595763683319091796875;     // nextafter(1,0)
	return r;
}

__device__ __forceinline__ Attempt attempt(uint4 w) {
	Attempt a;
	a.x = __dadd_rn(__dmul_rn(2.0, canonical(w.x, w.y)), -1.0);
	a.y = __dadd_rn(__dmul_rn(2.0, canonical(w.z, w.w)), -1.0);
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
// Batched form: every surface's polar transform in three launches.  Global
// block g belongs to the surface whose [block_base, next block_base) range
// holds it (binary search over the surface table).
namespace armab {
namespace {

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

__global__ void __launch_bounds__(kThreads)
noise_count_batch_kernel(const NoiseJob* __restrict__ jobs, int njobs, int* __restrict__ counts) {
	const NoiseJob& jb = jobs[find_job(jobs, njobs, blockIdx.x)];
	const unsigned long long lb = blockIdx.x - jb.block_base;
	const unsigned long long a0 = lb * kPerBlock + (unsigned long long)threadIdx.x * kPerThread;
	int cnt = 0;
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		const unsigned long long a = a0 + k;
		if (a < jb.n_attempts) cnt += attempt(jb.words[a]).ok ? 1 : 0;
	}
	int total;
	block_exclusive_scan(cnt, &total);
	if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads)
scan_counts_batch_kernel(const NoiseJob* __restrict__ jobs, const int* __restrict__ counts,
                         long long* __restrict__ offsets, long long* __restrict__ pairs) {
	const NoiseJob& jb = jobs[blockIdx.x];
	__shared__ long long carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (int base = 0; base < jb.nblocks; base += kThreads) {
		const int i = base + threadIdx.x;
		const int v = i < jb.nblocks ? counts[jb.block_base + i] : 0;
		int tot;
		const int ex = block_exclusive_scan(v, &tot);
		if (i < jb.nblocks) offsets[jb.block_base + i] = carry + ex;
		__syncthreads();
		if (threadIdx.x == 0) carry += tot;
		__syncthreads();
	}
	if (threadIdx.x == 0) pairs[blockIdx.x] = carry;
}

template <class T>
__global__ void __launch_bounds__(kThreads)
noise_scatter_batch_kernel(const NoiseJob* __restrict__ jobs, int njobs,
                           const long long* __restrict__ offsets) {
	const NoiseJob& jb = jobs[find_job(jobs, njobs, blockIdx.x)];
	const unsigned long long lb = blockIdx.x - jb.block_base;
	const unsigned long long a0 = lb * kPerBlock + (unsigned long long)threadIdx.x * kPerThread;
	T* out = static_cast<T*>(jb.out);
	Attempt at[kPerThread];
	int cnt = 0;
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		const unsigned long long a = a0 + k;
		if (a < jb.n_attempts) {
			at[k] = attempt(jb.words[a]);
		} else {
			at[k].ok = false;
		}
		cnt += at[k].ok ? 1 : 0;
	}
	int total;
	long long rank = offsets[blockIdx.x] + block_exclusive_scan(cnt, &total);
#pragma unroll
	for (int k = 0; k < kPerThread; ++k) {
		if (!at[k].ok) continue;
		const unsigned long long i0 = 2ull * (unsigned long long)rank;
		if (i0 < jb.n) {
			const double m = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(at[k].r2)), at[k].r2));
			out[i0] = T(__dadd_rn(__dmul_rn(__dmul_rn(at[k].y, m), jb.stddev), 0.0));
			if (i0 + 1 < jb.n)
				out[i0 + 1] = T(__dadd_rn(__dmul_rn(__dmul_rn(at[k].x, m), jb.stddev), 0.0));
			if (jb.attempts && i0 + 2 == jb.n) *jb.attempts = a0 + k + 1;
		}
		++rank;
	}
}

}  // namespace

void enqueue_white_noise_batch(Ctx* c, const std::vector<NoiseSpec>& specs, int precision,
                               long long* d_pairs) {
	ProfScope prof_(c, "noise");
	std::vector<NoiseJob> jobs(specs.size());
	long long total_blocks = 0;
	for (size_t k = 0; k < specs.size(); ++k) {
		const uint64_t na = specs[k].n_words / 4;
		const long long nb = (long long)std::max<uint64_t>(1, (na + kPerBlock - 1) / kPerBlock);
		ARMA_REQUIRE(!specs[k].attempts || specs[k].n % 2 == 0, ARMA_EINVAL,
		             "a noise chunk that continues a stream needs an even count");
		jobs[k] = NoiseJob{reinterpret_cast<const uint4*>(specs[k].words), na, specs[k].n,
		                   specs[k].stddev, specs[k].out, specs[k].attempts, int(total_blocks),
		                   int(nb)};
		total_blocks += nb;
	}
	ARMA_REQUIRE(total_blocks < (1ll << 31), ARMA_EINVAL, "white noise batch too large");
	if (jobs.empty()) return;
	auto* d_jobs = static_cast<NoiseJob*>(scratch_take(c, sizeof(NoiseJob) * jobs.size()));
	int* counts = static_cast<int*>(scratch_take(c, sizeof(int) * total_blocks));
	long long* offsets = static_cast<long long*>(scratch_take(c, sizeof(long long) * total_blocks));
	ARMA_CUDA_TRY(copy_async(c, d_jobs, jobs.data(), sizeof(NoiseJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	const int nj = int(jobs.size());
	noise_count_batch_kernel<<<int(total_blocks), kThreads, 0, c->stream>>>(d_jobs, nj, counts);
	scan_counts_batch_kernel<<<nj, kThreads, 0, c->stream>>>(d_jobs, counts, offsets, d_pairs);
	if (precision == ARMA_FP64)
		noise_scatter_batch_kernel<double><<<int(total_blocks), kThreads, 0, c->stream>>>(
		    d_jobs, nj, offsets);
	else
		noise_scatter_batch_kernel<float><<<int(total_blocks), kThreads, 0, c->stream>>>(
		    d_jobs, nj, offsets);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 3;
}

}  // namespace armab
