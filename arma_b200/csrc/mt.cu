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
// arithmetic in 32-bit integers.  The results are bit-identical to the
// sequential generator.
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr int kRingBits = 12;
constexpr int kRing = 1 << kRingBits;  // ring of raw words, >= nn + (nn-mm)
constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t temper(uint32_t y, const arma_mt_params& p) {
	y ^= y >> p.shift0;
	y ^= (y << p.shiftB) & p.maskB;
	y ^= (y << p.shiftC) & p.maskC;
	y ^= y >> p.shift1;
	return y;
}

__global__ void __launch_bounds__(kThreads)
mt_generate_kernel(const MtJob* __restrict__ jobs) {
	__shared__ uint32_t ring[kRing];
	const arma_mt_params p = jobs[blockIdx.x].p;
	const uint32_t seed = jobs[blockIdx.x].seed;
	const unsigned long long offset = jobs[blockIdx.x].offset;
	const unsigned long long count = jobs[blockIdx.x].count;
	uint32_t* __restrict__ out = jobs[blockIdx.x].out;
	const int n = p.nn, m = p.mm;
	const int chunk = n - m;
	if (threadIdx.x == 0) {
		// sgenrand_mt: Knuth's 1812433253 initialisation masked by wmask.
		uint32_t s = seed;
		for (int k = 0; k < n; ++k) {
			ring[k] = s & p.wmask;
			s = 1812433253u * (s ^ (s >> 30)) + uint32_t(k + 1);
		}
	}
	__syncthreads();
	const unsigned long long end = (unsigned long long)n + offset + count;
	const uint32_t mask = kRing - 1;
	auto compute = [&](unsigned long long j0) {
		for (int t = threadIdx.x; t < chunk; t += blockDim.x) {
			const unsigned long long j = j0 + t;
			if (j < end) {
				const uint32_t y = (ring[(j - n) & mask] & p.umask) |
				                   (ring[(j - n + 1) & mask] & p.lmask);
				ring[j & mask] = ring[(j - n + m) & mask] ^ (y >> 1) ^ ((y & 1u) ? p.aaa : 0u);
			}
		}
	};
	unsigned long long j0 = n;
	compute(j0);
	__syncthreads();
	while (j0 < end) {
		for (int t = threadIdx.x; t < chunk; t += blockDim.x) {
			const unsigned long long j = j0 + t;
			if (j < end) {
				const unsigned long long w = j - n;  // output word index
				if (w >= offset) out[w - offset] = temper(ring[j & mask], p);
			}
		}
		compute(j0 + chunk);
		__syncthreads();
		j0 += chunk;
	}
}

}  // namespace

void launch_mt_generate_batch(Ctx* c, const std::vector<MtJob>& jobs) {
	ProfScope prof_(c, "mt");
	for (const MtJob& j : jobs) {
		ARMA_REQUIRE(j.p.nn > 1 && j.p.mm > 0 && j.p.mm < j.p.nn, ARMA_EINVAL,
		             "bad MT parameter set");
		ARMA_REQUIRE(j.p.nn + (j.p.nn - j.p.mm) <= kRing, ARMA_EINVAL,
		             "MT state too large for the device generator");
	}
	if (jobs.empty()) return;
	MtJob* d_jobs = static_cast<MtJob*>(scratch_take(c, sizeof(MtJob) * jobs.size()));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(MtJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	mt_generate_kernel<<<int(jobs.size()), kThreads, 0, c->stream>>>(d_jobs);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

void launch_mt_generate(Ctx* c, const arma_mt_params& p, uint32_t seed,
                        uint64_t offset, uint64_t n, uint32_t* d_out) {
	if (n == 0) return;
	launch_mt_generate_batch(c, {MtJob{p, seed, offset, n, d_out}});
	// the job table lives in scratch: keep it alive until the kernel has read it
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
}

}  // namespace armab
