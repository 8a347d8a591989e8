// The moving-average filter: zeta = eps - sum_{m != 0} theta(m) eps(n - m),
// a causal 3-D FIR over the white noise with zero history.
//
// Reference: MA_model::generate_surface (src/generator/ma_model.cc:42-61)
// convolves the noise with the kernel K = -theta, K(0,0,0) = 1, by FFT
// overlap-add (src/apmath/convolution.hh:58-130), which is the causal linear
// convolution truncated to the surface; the reference's own test writes the
// same sum directly (src/test/convolution-test.cc:17-50).  Here it is the
// direct sum on the CUDA cores: with no feedback the filter is data-parallel
// and compute-bound (2 P FLOP per point for P taps), and at the reference's
// orders (up to a few thousand taps) the direct form needs one pass over the
// noise where an FFT form needs several over padded complex arrays.
//
// A block owns a tile of 8 time steps x 16 rows (x) x 16 R columns (y); each
// thread owns R columns (y = lane + 16 r) of one row at each of the 8 time
// steps, 8 R accumulators.  The block streams the noise slices its outputs
// depend on (latest first) through two shared-memory buffers filled by
// cp.async (zero fill outside the surface: the zero history), and every slice
// feeds each of the 8 time steps with its own lag k = t - s.  Taps live in the
// kernel's parameter block (constant bank: a broadcast operand that does not
// use the shared-memory data path); more taps than one parameter block holds
// run as several launches over ranges of (k, i) tap rows, each adding into
// the output.
#include <algorithm>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr int kMaTT = 8;           // time steps per block
constexpr int kMaThreads = 256;    // 16 (y lanes) x 16 (x rows)
constexpr int kMaParamBytes = 30720;
constexpr int kMaSmemLimit = 227 * 1024;

__device__ __forceinline__ double ma_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float ma_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <class T, int CAP>
struct MaTaps {
	T v[CAP];
};

template <class T>
struct MaShape;
template <>
struct MaShape<double> {
	static constexpr int R = 4;
};
template <>
struct MaShape<float> {
	static constexpr int R = 4;
};

// Shared-memory row pitch: the two x rows a warp reads sit in disjoint bank
// halves for 4-byte elements (pitch = 16 mod 32 words).
template <class T>
__host__ __device__ inline int ma_pitch(int cols) {
	if (sizeof(T) == 4) return cols + ((16 - cols % 32) + 32) % 32;
	return cols;
}

template <class T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
	const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
	const int n = valid ? int(sizeof(T)) : 0;
	if (sizeof(T) == 8)
		asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n)
		             : "memory");
	else
		asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n)
		             : "memory");
}

template <class T, int CAP>
__global__ void __launch_bounds__(kMaThreads)
ma_fir_kernel(const T* __restrict__ eps, T* __restrict__ zeta, int nt, int nx, int ny, int px,
              int py, int r0, int r1, int accumulate, const __grid_constant__ MaTaps<T, CAP> taps) {
	constexpr int R = MaShape<T>::R, TT = kMaTT, TY = 16 * R, TX = 16;
	extern __shared__ __align__(16) unsigned char ma_smem[];
	T* sbuf = reinterpret_cast<T*>(ma_smem);
	const int rows = TX + px - 1, cols = TY + py - 1, ld = ma_pitch<T>(cols);
	const int tile = rows * ld;
	const int y0 = blockIdx.x * TY, x0 = blockIdx.y * TX, t0 = blockIdx.z * TT;
	const int lane = threadIdx.x, xl = threadIdx.y, tid = xl * 16 + lane;
	const int kmin = r0 / px, kmax = (r1 - 1) / px;
	const int s_hi = min(nt - 1, t0 + TT - 1 - kmin), s_lo = max(0, t0 - kmax);
	const size_t plane = size_t(nx) * ny;

	T acc[TT][R];
#pragma unroll
	for (int tt = 0; tt < TT; ++tt)
#pragma unroll
		for (int r = 0; r < R; ++r) acc[tt][r] = T(0);

	auto load = [&](int s, T* dst) {
		const T* src = eps + size_t(s) * plane;
		for (int idx = tid; idx < rows * cols; idx += kMaThreads) {
			const int rr = idx / cols, cc = idx - rr * cols;
			const int gx = x0 - (px - 1) + rr, gy = y0 - (py - 1) + cc;
			const bool ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
			cp_async_elem(dst + rr * ld + cc, ok ? src + size_t(gx) * ny + gy : eps, ok);
		}
		asm volatile("cp.async.commit_group;" ::: "memory");
	};

	if (s_hi >= s_lo) {
		load(s_hi, sbuf);
		int b = 0;
		for (int s = s_hi; s >= s_lo; --s, b ^= 1) {
			if (s > s_lo) load(s - 1, sbuf + (b ^ 1) * tile);
			else asm volatile("cp.async.commit_group;" ::: "memory");
			asm volatile("cp.async.wait_group 1;" ::: "memory");
			__syncthreads();
			const T* buf = sbuf + b * tile;
			for (int i = 0; i < px; ++i) {
				// active time steps of this (slice, tap row): k = t - s, row k px + i
				// inside [r0, r1), t inside the surface (uniform over the block)
				bool on[TT];
				int base[TT];
#pragma unroll
				for (int tt = 0; tt < TT; ++tt) {
					const int row = (t0 + tt - s) * px + i;
					on[tt] = t0 + tt < nt && t0 + tt >= s && row >= r0 && row < r1;
					base[tt] = (row - r0) * py;
				}
				const T* srow = buf + (xl + px - 1 - i) * ld + lane + py - 1;
				for (int j = 0; j < py; ++j) {
					T v[R];
#pragma unroll
					for (int r = 0; r < R; ++r) v[r] = srow[16 * r - j];
#pragma unroll
					for (int tt = 0; tt < TT; ++tt) {
						if (on[tt]) {
							const T c = taps.v[base[tt] + j];
#pragma unroll
							for (int r = 0; r < R; ++r) acc[tt][r] = ma_fma(c, v[r], acc[tt][r]);
						}
					}
				}
			}
			__syncthreads();
		}
	}
	const int x = x0 + xl;
	if (x >= nx) return;
#pragma unroll
	for (int tt = 0; tt < TT; ++tt) {
		const int t = t0 + tt;
		if (t >= nt) break;
#pragma unroll
		for (int r = 0; r < R; ++r) {
			const int y = y0 + lane + 16 * r;
			if (y >= ny) continue;
			T* p = zeta + size_t(t) * plane + size_t(x) * ny + y;
			*p = accumulate ? *p + acc[tt][r] : acc[tt][r];
		}
	}
}

template <class T>
size_t ma_smem_bytes(int px, int py) {
	constexpr int R = MaShape<T>::R;
	const int rows = 16 + px - 1, cols = 16 * R + py - 1;
	return 2 * size_t(rows) * ma_pitch<T>(cols) * sizeof(T);
}

template <class T, int CAP>
void launch_chunks(Ctx* c, const std::vector<T>& K, const int order[3], const int shape[3],
                   const T* eps, T* zeta) {
	constexpr int R = MaShape<T>::R;
	const int pt = order[0], px = order[1], py = order[2];
	const int rows_total = pt * px;
	const int rows_per = std::max(1, CAP / py);
	const size_t smem = ma_smem_bytes<T>(px, py);
	ARMA_CUDA_TRY(cudaFuncSetAttribute(ma_fir_kernel<T, CAP>,
	                                   cudaFuncAttributeMaxDynamicSharedMemorySize, kMaSmemLimit));
	const dim3 grid((shape[2] + 16 * R - 1) / (16 * R), (shape[1] + 15) / 16,
	                (shape[0] + kMaTT - 1) / kMaTT);
	ARMA_REQUIRE(grid.y <= 65535 && grid.z <= 65535, ARMA_EINVAL, "surface too large");
	for (int r0 = 0; r0 < rows_total; r0 += rows_per) {
		const int r1 = std::min(rows_total, r0 + rows_per);
		MaTaps<T, CAP> taps;
		std::fill(taps.v, taps.v + CAP, T(0));
		std::copy(K.begin() + size_t(r0) * py, K.begin() + size_t(r1) * py, taps.v);
		ma_fir_kernel<T, CAP><<<grid, dim3(16, 16), smem, c->stream>>>(
		    eps, zeta, shape[0], shape[1], shape[2], px, py, r0, r1, r0 > 0 ? 1 : 0, taps);
		ARMA_CUDA_TRY(cudaGetLastError());
		++c->launches;
	}
}

template <class T>
void ma_filter_impl(Ctx* c, const double* theta, const int order[3], const int shape[3],
                    const T* eps, T* zeta) {
	const size_t P = size_t(order[0]) * order[1] * order[2];
	ARMA_REQUIRE(ma_smem_bytes<T>(order[1], order[2]) <= size_t(kMaSmemLimit), ARMA_ENOTSUP,
	             "MA order too wide in x/y for the shared-memory tile");
	// K = -theta with K(0,0,0) = 1 (src/generator/ma_model.cc:55-58)
	std::vector<T> K(P);
	K[0] = T(1);
	for (size_t q = 1; q < P; ++q) K[q] = T(-theta[q]);
	constexpr int kSmall = 512;
	constexpr int kLarge = kMaParamBytes / int(sizeof(T));
	if (P <= size_t(kSmall)) launch_chunks<T, kSmall>(c, K, order, shape, eps, zeta);
	else launch_chunks<T, kLarge>(c, K, order, shape, eps, zeta);
}

}  // namespace

void launch_ma_filter(Ctx* c, const double* theta, const int order[3], const int shape[3],
                      int precision, const void* d_eps, void* d_zeta) {
	ProfScope prof_(c, "ma_fir");
	if (precision == ARMA_FP64)
		ma_filter_impl(c, theta, order, shape, static_cast<const double*>(d_eps),
		               static_cast<double*>(d_zeta));
	else
		ma_filter_impl(c, theta, order, shape, static_cast<const float*>(d_eps),
		               static_cast<float*>(d_zeta));
}

}  // namespace armab
