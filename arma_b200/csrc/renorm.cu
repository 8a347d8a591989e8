// Variance renormalisation of a generated surface.
//
// The reference scales the surface by sqrt(acf(0,0,0) / var) where var is
// taken through stats::variance(Array) = gsl_stats_variance(view.data(), 1,
// view.numElements()) on the view zeta(shape/2 : shape-1)
// (src/generator/basic_arma_model.cc:102-106, src/stats/statistics.hh:35-44):
// numElements() contiguous values starting at the view's first element.  The
// unbiased variance is computed here in FP64 by a deterministic two-pass
// reduction (mean, then sum of squared deviations), and the scale stays on
// the device so the multiply needs no host round trip.
#include <algorithm>

#include "internal.h"

namespace armab {
namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 592;  // 4 per SM on 148 SMs

template <class T>
__global__ void __launch_bounds__(kThreads)
partial_sum_kernel(const T* __restrict__ x, unsigned long long n,
                   const double* __restrict__ mean, double* __restrict__ partial) {
	__shared__ double sh[kThreads / 32];
	const double m = mean ? *mean : 0.0;
	double acc = 0.0;
	for (unsigned long long i = blockIdx.x * (unsigned long long)kThreads + threadIdx.x; i < n;
	     i += (unsigned long long)gridDim.x * kThreads) {
		const double v = double(x[i]);
		if (mean) {
			const double d = v - m;
			acc = fma(d, d, acc);
		} else {
			acc += v;
		}
	}
	for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
	if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x == 0) {
		double s = 0.0;
		for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
		partial[blockIdx.x] = s;
	}
}

// Fixed-order sum of the block partials.  mode 0: mean = sum / n;
// mode 1: scale = sqrt(acf0 / (sum / (n-1))).
__global__ void finish_kernel(const double* __restrict__ partial, int nb,
                              unsigned long long n, int mode, double acf0,
                              double* __restrict__ out) {
	__shared__ double sh[32];
	double s = 0.0;
	for (int i = threadIdx.x; i < nb; i += 32) s += partial[i];
	sh[threadIdx.x] = s;
	__syncwarp();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int i = 0; i < 32; ++i) t += sh[i];
		if (mode == 0) *out = t / double(n);
		else *out = sqrt(acf0 / (t / double(n - 1)));
	}
}

template <class T>
__global__ void __launch_bounds__(kThreads)
scale_kernel(T* __restrict__ x, unsigned long long n, const double* __restrict__ scale) {
	const double s = *scale;
	for (unsigned long long i = blockIdx.x * (unsigned long long)kThreads + threadIdx.x; i < n;
	     i += (unsigned long long)gridDim.x * kThreads)
		x[i] = T(double(x[i]) * s);
}

template <class T>
void renorm_impl(Ctx* c, T* z, const int shape[3], double acf0, double* d_scale) {
	const long long nt = shape[0], nx = shape[1], ny = shape[2];
	const unsigned long long off = (unsigned long long)((nt / 2) * nx + nx / 2) * ny + ny / 2;
	const unsigned long long cnt =
	    (unsigned long long)(nt - nt / 2) * (nx - nx / 2) * (ny - ny / 2);
	const unsigned long long n = (unsigned long long)nt * nx * ny;
	ARMA_REQUIRE(cnt >= 2, ARMA_EINVAL, "surface too small for variance renormalisation");
	double* partial = static_cast<double*>(scratch_take(c, sizeof(double) * kBlocks));
	double* mean = static_cast<double*>(scratch_take(c, sizeof(double)));
	partial_sum_kernel<T><<<kBlocks, kThreads, 0, c->stream>>>(z + off, cnt, nullptr, partial);
	finish_kernel<<<1, 32, 0, c->stream>>>(partial, kBlocks, cnt, 0, acf0, mean);
	partial_sum_kernel<T><<<kBlocks, kThreads, 0, c->stream>>>(z + off, cnt, mean, partial);
	finish_kernel<<<1, 32, 0, c->stream>>>(partial, kBlocks, cnt, 1, acf0, d_scale);
	scale_kernel<T><<<kBlocks, kThreads, 0, c->stream>>>(z, n, d_scale);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 5;
}

}  // namespace

void launch_renorm(Ctx* c, void* d_zeta, const int shape[3], int precision,
                   double acf0, double* d_scale) {
	ProfScope prof_(c, "renorm");
	if (precision == ARMA_FP64)
		renorm_impl(c, static_cast<double*>(d_zeta), shape, acf0, d_scale);
	else
		renorm_impl(c, static_cast<float*>(d_zeta), shape, acf0, d_scale);
}

}  // namespace armab

// ---------------------------------------------------------------------------
// Batched form: the renormalisation of many surfaces in five launches.
namespace armab {
namespace {

constexpr int kBatchBlocks = 32;  // partial sums per surface

struct RenormJob {
	void* z;
	unsigned long long off, cnt, n;
	double acf0;
	double* scale;
	const void* lut;  // NIT coefficient table (nit_lut_coefficients) after the scale, or null
	int lut_nodes;
	int vec;          // z is 16-byte aligned: 16-byte accesses
	double lut_x0, lut_inv_dx;
};

template <class T>
__global__ void __launch_bounds__(kThreads)
partial_batch_kernel(const RenormJob* __restrict__ jobs, const double* __restrict__ means,
                     double* __restrict__ partial) {
	__shared__ double sh[kThreads / 32];
	const int s = blockIdx.x / kBatchBlocks, b = blockIdx.x % kBatchBlocks;
	const RenormJob& jb = jobs[s];
	const T* x = static_cast<const T*>(jb.z) + jb.off;
	const double m = means ? means[s] : 0.0;
	double acc = 0.0;
	// the thread's values in index order, kUnroll loads in flight at a time
	constexpr int kUnroll = 8;
	const unsigned long long stride = (unsigned long long)kBatchBlocks * kThreads;
	for (unsigned long long i0 = (unsigned long long)b * kThreads + threadIdx.x; i0 < jb.cnt;
	     i0 += stride * kUnroll) {
		T v[kUnroll];
#pragma unroll
		for (int r = 0; r < kUnroll; ++r) {
			const unsigned long long i = i0 + r * stride;
			v[r] = i < jb.cnt ? x[i] : T(0);
		}
#pragma unroll
		for (int r = 0; r < kUnroll; ++r) {
			if (i0 + r * stride >= jb.cnt) break;
			if (means) {
				const double d = double(v[r]) - m;
				acc = fma(d, d, acc);
			} else {
				acc += double(v[r]);
			}
		}
	}
	for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
	if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
		partial[blockIdx.x] = t;
	}
}

__global__ void finish_batch_kernel(const RenormJob* __restrict__ jobs,
                                    const double* __restrict__ partial, int mode,
                                    double* __restrict__ means) {
	const RenormJob& jb = jobs[blockIdx.x];
	if (threadIdx.x != 0) return;
	double t = 0.0;
	for (int i = 0; i < kBatchBlocks; ++i) t += partial[blockIdx.x * kBatchBlocks + i];
	if (mode == 0) means[blockIdx.x] = t / double(jb.cnt);
	else *jb.scale = sqrt(jb.acf0 / (t / double(jb.cnt - 1)));
}

// Blocks in proportion to each surface's points (kScaleChunk elements per
// block, kLutChunks times that for a surface with a NIT table, whose block
// first stages the table in shared memory), so that the largest surfaces do
// not trail; block b belongs to the last job whose first block is <= b.
constexpr int kScaleChunk = kThreads * 16;
constexpr int kLutChunks = 16;
constexpr size_t kLutSmemMax = 48 * 1024;

template <class T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };

// zeta *= scale, then (when the job has one) the NIT table: one read and one
// write per value, 16-byte accesses where the surface is aligned.  lut_smem:
// the launch's dynamic shared memory holds a job's table (else it is read
// through L1).
template <class T>
__global__ void __launch_bounds__(kThreads)
scale_batch_kernel(const RenormJob* __restrict__ jobs, const int* __restrict__ first_block,
                   int njobs, int lut_smem) {
	using Coef = typename NitCoef<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	int lo = 0, hi = njobs - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) / 2;
		if (first_block[mid] <= int(blockIdx.x)) lo = mid; else hi = mid - 1;
	}
	const RenormJob& jb = jobs[lo];
	T* x = static_cast<T*>(jb.z);
	const double sc = *jb.scale;
	const Coef* lut = static_cast<const Coef*>(jb.lut);
	const int nodes = jb.lut_nodes;
	const T x0 = T(jb.lut_x0), inv_dx = T(jb.lut_inv_dx);
	if (lut && lut_smem) {
		Coef* st = reinterpret_cast<Coef*>(smem_raw);
		for (int i = threadIdx.x; i <= nodes; i += kThreads) st[i] = lut[i];
		__syncthreads();
		lut = st;
	}
	auto map = [&](T v) {
		v = T(double(v) * sc);
		return lut ? nit_lut_map(v, lut, nodes, x0, inv_dx) : v;
	};
	const int chunks = lut ? kLutChunks : 1;
	for (int ch = 0; ch < chunks; ++ch) {
		const unsigned long long i0 =
		    ((unsigned long long)(blockIdx.x - first_block[lo]) * chunks + ch) * kScaleChunk;
		if (i0 >= jb.n) break;
		const unsigned long long i1 = min(jb.n, i0 + kScaleChunk);
		if (jb.vec) {
			// every thread's kPer vectors of the chunk are loaded before any is
			// mapped, so that they are all in flight at once
			using V = typename Vec16<T>::type;
			constexpr int W = Vec16<T>::n;
			constexpr int kPer = kScaleChunk / (W * kThreads);
			const unsigned long long nv = (i1 - i0) / W;  // i0 is a multiple of kScaleChunk
			V* xv = reinterpret_cast<V*>(x + i0);
			V v[kPer];
#pragma unroll
			for (int r = 0; r < kPer; ++r) {
				const unsigned long long i = threadIdx.x + (unsigned long long)r * kThreads;
				if (i < nv) v[r] = xv[i];
			}
#pragma unroll
			for (int r = 0; r < kPer; ++r) {
				const unsigned long long i = threadIdx.x + (unsigned long long)r * kThreads;
				if (i < nv) {
					T* e = reinterpret_cast<T*>(&v[r]);
#pragma unroll
					for (int k = 0; k < W; ++k) e[k] = map(e[k]);
					xv[i] = v[r];
				}
			}
			for (unsigned long long i = i0 + nv * W + threadIdx.x; i < i1; i += kThreads)
				x[i] = map(x[i]);
		} else {
			for (unsigned long long i = i0 + threadIdx.x; i < i1; i += kThreads) x[i] = map(x[i]);
		}
	}
}

}  // namespace

void launch_renorm_batch(Ctx* c, const std::vector<RenormSpec>& specs, int precision,
                         bool apply) {
	ProfScope prof_(c, "renorm");
	if (specs.empty()) return;
	std::vector<RenormJob> jobs(specs.size());
	for (size_t k = 0; k < specs.size(); ++k) {
		const long long nt = specs[k].shape[0], nx = specs[k].shape[1], ny = specs[k].shape[2];
		RenormJob& j = jobs[k];
		j.z = specs[k].z;
		j.off = (unsigned long long)((nt / 2) * nx + nx / 2) * ny + ny / 2;
		j.cnt = (unsigned long long)(nt - nt / 2) * (nx - nx / 2) * (ny - ny / 2);
		j.n = (unsigned long long)nt * nx * ny;
		j.acf0 = specs[k].acf0;
		j.scale = specs[k].d_scale;
		j.lut = specs[k].lut;
		j.lut_nodes = specs[k].lut_nodes;
		j.lut_x0 = specs[k].lut_x0;
		j.lut_inv_dx = specs[k].lut_inv_dx;
		j.vec = (reinterpret_cast<uintptr_t>(j.z) % 16) == 0;
		ARMA_REQUIRE(!j.lut || j.lut_nodes >= 4, ARMA_EINVAL, "NIT table needs at least 4 nodes");
		ARMA_REQUIRE(j.cnt >= 2, ARMA_EINVAL, "surface too small for variance renormalisation");
	}
	const int ns = int(jobs.size());
	std::vector<int> first(ns);
	int sblocks = 0, max_nodes = 0;
	for (int k = 0; k < ns; ++k) {
		first[k] = sblocks;
		const unsigned long long chunk =
		    (unsigned long long)kScaleChunk * (jobs[k].lut ? kLutChunks : 1);
		sblocks += int((jobs[k].n + chunk - 1) / chunk);
		if (jobs[k].lut) max_nodes = std::max(max_nodes, jobs[k].lut_nodes);
	}
	// the largest table of the launch in shared memory when it fits
	const size_t coef_bytes = precision == ARMA_FP64 ? sizeof(double4) : sizeof(float4);
	size_t lut_smem = max_nodes ? coef_bytes * (size_t(max_nodes) + 1) : 0;
	if (lut_smem > kLutSmemMax) lut_smem = 0;
	int* d_first = static_cast<int*>(scratch_take(c, sizeof(int) * ns));
	ARMA_CUDA_TRY(copy_async(c, d_first, first.data(), sizeof(int) * ns, cudaMemcpyHostToDevice,
	                              c->stream));
	auto* d_jobs = static_cast<RenormJob*>(scratch_take(c, sizeof(RenormJob) * jobs.size()));
	double* partial = static_cast<double*>(scratch_take(c, sizeof(double) * ns * kBatchBlocks));
	double* means = static_cast<double*>(scratch_take(c, sizeof(double) * ns));
	ARMA_CUDA_TRY(copy_async(c, d_jobs, jobs.data(), sizeof(RenormJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	const int g = ns * kBatchBlocks;
	if (precision == ARMA_FP64) {
		partial_batch_kernel<double><<<g, kThreads, 0, c->stream>>>(d_jobs, nullptr, partial);
		finish_batch_kernel<<<ns, 32, 0, c->stream>>>(d_jobs, partial, 0, means);
		partial_batch_kernel<double><<<g, kThreads, 0, c->stream>>>(d_jobs, means, partial);
		finish_batch_kernel<<<ns, 32, 0, c->stream>>>(d_jobs, partial, 1, means);
		if (apply)
			scale_batch_kernel<double><<<sblocks, kThreads, lut_smem, c->stream>>>(d_jobs, d_first,
			                                                                        ns, lut_smem > 0);
	} else {
		partial_batch_kernel<float><<<g, kThreads, 0, c->stream>>>(d_jobs, nullptr, partial);
		finish_batch_kernel<<<ns, 32, 0, c->stream>>>(d_jobs, partial, 0, means);
		partial_batch_kernel<float><<<g, kThreads, 0, c->stream>>>(d_jobs, means, partial);
		finish_batch_kernel<<<ns, 32, 0, c->stream>>>(d_jobs, partial, 1, means);
		if (apply)
			scale_batch_kernel<float><<<sblocks, kThreads, lut_smem, c->stream>>>(d_jobs, d_first, ns,
			                                                                       lut_smem > 0);
	}
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += apply ? 5 : 4;
}

}  // namespace armab
