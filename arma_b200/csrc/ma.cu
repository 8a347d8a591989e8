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
// A block owns a tile of 8 time steps x 16 rows (x) x 16 R columns (y), R = 4
// for FP64 and 8 for FP32 (register budget: 2 blocks of 256 threads per SM); each
// thread owns R columns (y = lane + 16 r) of one row at each of the 8 time
// steps, 8 R accumulators.  The block streams the noise slices its outputs
// depend on (latest first) through two shared-memory buffers filled by
// cp.async (zero fill outside the surface: the zero history); with each slice
// s it stages the taps every time step needs from it, c(i, j, tt) =
// K(t0 + tt - s, i, j) (zero where the lag falls outside the order), so the
// inner loop is branch-free: per (i, j) R noise values and 8 taps from shared
// memory feed 8 R FMAs (4 R on slices that reach only one half of the time
// steps).  Orders whose tap block does not fit run as several
// launches over ranges of i, each adding into the output.
#include <algorithm>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

constexpr int kMaTT = 8;           // time steps per block
constexpr int kMaThreads = 256;    // 16 (y lanes) x 16 (x rows)
constexpr int kMaSmemLimit = 227 * 1024;
constexpr int kMaTapBytes = 64 * 1024;  // both tap buffers of one launch

__device__ __forceinline__ double ma_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float ma_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <class T>
struct MaShape;
template <>
struct MaShape<double> {
	static constexpr int R = 4;
};
template <>
struct MaShape<float> {
	static constexpr int R = 8;
};

// Shared-memory row pitch: the two x rows a warp reads sit in disjoint bank
// halves for 4-byte elements (pitch = 16 mod 32 words).
template <class T>
__host__ __device__ inline int ma_pitch(int cols) {
	if (sizeof(T) == 4) return cols + ((16 - cols % 32) + 32) % 32;
	return cols;
}

// Elements of one noise tile, rounded up to 16 bytes.
template <class T>
__host__ __device__ inline int ma_tile_elems(int px, int py) {
	constexpr int R = MaShape<T>::R;
	const int n = (16 + px - 1) * ma_pitch<T>(16 * R + py - 1);
	constexpr int q = 16 / int(sizeof(T));
	return (n + q - 1) / q * q;
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

// N taps of one (i, j) (time steps TB .. TB+N-1), from 16-byte aligned
// shared memory.
template <int N>
__device__ __forceinline__ void load_taps(const double* p, double (&c)[kMaTT]) {
#pragma unroll
	for (int q = 0; q < N / 2; ++q) {
		const double2 v = reinterpret_cast<const double2*>(p)[q];
		c[2 * q] = v.x;
		c[2 * q + 1] = v.y;
	}
}
template <int N>
__device__ __forceinline__ void load_taps(const float* p, float (&c)[kMaTT]) {
#pragma unroll
	for (int q = 0; q < N / 4; ++q) {
		const float4 v = reinterpret_cast<const float4*>(p)[q];
		c[4 * q] = v.x;
		c[4 * q + 1] = v.y;
		c[4 * q + 2] = v.z;
		c[4 * q + 3] = v.w;
	}
}

// One slice's contribution to the time steps TB .. TB+TN-1 (the others have
// no tap on this slice).
template <class T, int R, int TB, int TN>
__device__ __forceinline__ void ma_slice(T (&acc)[kMaTT][R], const T* buf, const T* cb, int ld,
                                         int xl, int lane, int px, int py, int i0, int ni) {
	for (int i = 0; i < ni; ++i) {
		const T* srow = buf + (xl + px - 1 - (i0 + i)) * ld + lane + py - 1;
		const T* crow = cb + i * py * kMaTT + TB;
#pragma unroll 2
		for (int j = 0; j < py; ++j) {
			T v[R], c[kMaTT];
#pragma unroll
			for (int r = 0; r < R; ++r) v[r] = srow[16 * r - j];
			load_taps<TN>(crow + j * kMaTT, c);
#pragma unroll
			for (int tt = 0; tt < TN; ++tt)
#pragma unroll
				for (int r = 0; r < R; ++r)
					acc[TB + tt][r] = ma_fma(c[tt], v[r], acc[TB + tt][r]);
		}
	}
}

template <class T>
__global__ void __launch_bounds__(kMaThreads)
ma_fir_kernel(const T* __restrict__ eps, T* __restrict__ zeta, const T* __restrict__ K, int nt,
              int nx, int ny, int pt, int px, int py, int i0, int i1, int accumulate) {
	constexpr int R = MaShape<T>::R, TT = kMaTT, TY = 16 * R, TX = 16;
	extern __shared__ __align__(16) unsigned char ma_smem[];
	const int rows = TX + px - 1, cols = TY + py - 1, ld = ma_pitch<T>(cols);
	const int tile = ma_tile_elems<T>(px, py);
	const int ni = i1 - i0, ctile = ni * py * TT;
	T* ebuf = reinterpret_cast<T*>(ma_smem);
	T* cbuf = ebuf + 2 * tile;
	const int y0 = blockIdx.x * TY, x0 = blockIdx.y * TX, t0 = blockIdx.z * TT;
	const int lane = threadIdx.x, xl = threadIdx.y, tid = xl * 16 + lane;
	const int s_hi = min(nt - 1, t0 + TT - 1), s_lo = max(0, t0 - (pt - 1));
	const size_t plane = size_t(nx) * ny;

	T acc[TT][R];
#pragma unroll
	for (int tt = 0; tt < TT; ++tt)
#pragma unroll
		for (int r = 0; r < R; ++r) acc[tt][r] = T(0);

	// noise slice s and its taps into buffer b, one cp.async group
	auto load = [&](int s, int b) {
		const T* src = eps + size_t(s) * plane;
		T* dst = ebuf + b * tile;
		for (int idx = tid; idx < rows * cols; idx += kMaThreads) {
			const int rr = idx / cols, cc = idx - rr * cols;
			const int gx = x0 - (px - 1) + rr, gy = y0 - (py - 1) + cc;
			const bool ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
			cp_async_elem(dst + rr * ld + cc, ok ? src + size_t(gx) * ny + gy : eps, ok);
		}
		T* cdst = cbuf + b * ctile;
		for (int idx = tid; idx < ctile; idx += kMaThreads) {
			const int tt = idx % TT, ij = idx / TT;
			const int j = ij % py, i = i0 + ij / py;
			const int k = t0 + tt - s;
			const bool ok = k >= 0 && k < pt && t0 + tt < nt;
			cp_async_elem(cdst + idx, ok ? K + (size_t(k) * px + i) * py + j : K, ok);
		}
		asm volatile("cp.async.commit_group;" ::: "memory");
	};

	load(s_hi, 0);
	int b = 0;
	for (int s = s_hi; s >= s_lo; --s, b ^= 1) {
		if (s > s_lo) load(s - 1, b ^ 1);
		else asm volatile("cp.async.commit_group;" ::: "memory");
		asm volatile("cp.async.wait_group 1;" ::: "memory");
		__syncthreads();
		const T* buf = ebuf + b * tile;
		const T* cb = cbuf + b * ctile;
		// time steps with a tap on slice s: lag t0 + tt - s in [0, pt)
		const int lo = max(0, s - t0), hi = min(min(TT, s - t0 + pt), nt - t0);
		if (lo >= TT / 2)
			ma_slice<T, R, TT / 2, TT / 2>(acc, buf, cb, ld, xl, lane, px, py, i0, ni);
		else if (hi <= TT / 2)
			ma_slice<T, R, 0, TT / 2>(acc, buf, cb, ld, xl, lane, px, py, i0, ni);
		else
			ma_slice<T, R, 0, TT>(acc, buf, cb, ld, xl, lane, px, py, i0, ni);
		__syncthreads();
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

// Rows of taps (values of i) per launch: both tap buffers within kMaTapBytes.
template <class T>
int ma_rows_per_launch(int px, int py) {
	const int per_row = 2 * py * kMaTT * int(sizeof(T));
	return std::max(1, std::min(px, kMaTapBytes / per_row));
}

template <class T>
size_t ma_smem_bytes(int px, int py) {
	const int ni = ma_rows_per_launch<T>(px, py);
	return (2 * size_t(ma_tile_elems<T>(px, py)) + 2 * size_t(ni) * py * kMaTT) * sizeof(T);
}

template <class T>
void ma_filter_impl(Ctx* c, const double* theta, const int order[3], const int shape[3],
                    const T* eps, T* zeta) {
	constexpr int R = MaShape<T>::R;
	const int pt = order[0], px = order[1], py = order[2];
	const size_t P = size_t(pt) * px * py;
	const size_t smem = ma_smem_bytes<T>(px, py);
	ARMA_REQUIRE(smem <= size_t(kMaSmemLimit), ARMA_ENOTSUP,
	             "MA order too wide in x/y for the shared-memory tile");
	// K = -theta with K(0,0,0) = 1 (src/generator/ma_model.cc:55-58)
	std::vector<T> K(P);
	K[0] = T(1);
	for (size_t q = 1; q < P; ++q) K[q] = T(-theta[q]);
	T* dK = static_cast<T*>(scratch_take(c, P * sizeof(T)));
	ARMA_CUDA_TRY(copy_async(c, dK, K.data(), P * sizeof(T), cudaMemcpyHostToDevice, c->stream));
	ARMA_CUDA_TRY(cudaFuncSetAttribute(ma_fir_kernel<T>,
	                                   cudaFuncAttributeMaxDynamicSharedMemorySize, kMaSmemLimit));
	const dim3 grid((shape[2] + 16 * R - 1) / (16 * R), (shape[1] + 15) / 16,
	                (shape[0] + kMaTT - 1) / kMaTT);
	ARMA_REQUIRE(grid.y <= 65535 && grid.z <= 65535, ARMA_EINVAL, "surface too large");
	const int rows_per = ma_rows_per_launch<T>(px, py);
	for (int i0 = 0; i0 < px; i0 += rows_per) {
		const int i1 = std::min(px, i0 + rows_per);
		ma_fir_kernel<T><<<grid, dim3(16, 16), smem, c->stream>>>(
		    eps, zeta, dK, shape[0], shape[1], shape[2], pt, px, py, i0, i1, i0 > 0 ? 1 : 0);
		ARMA_CUDA_TRY(cudaGetLastError());
		++c->launches;
	}
	// (a copy from pageable memory has been staged by the time cudaMemcpyAsync
	// returns, so K may go out of scope)
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
