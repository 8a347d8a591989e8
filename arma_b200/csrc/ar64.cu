// Plain FP64 AR filter with the reference's exact summation order.
//
// ar_generate_surface (reference src/generator/ar_model_surf.cc:5-36) updates
// zeta in place in C order; each point sums phi(k,i,j) * zeta(t-k,x-i,y-j)
// over k, i, j ascending (truncated at the array start) into a running sum
// that starts at 0, then adds the sum to the noise already stored at the
// point.  Every point depends only on points with smaller t+x+y, so all points
// of one hyperplane t+x+y = s are independent: one launch per hyperplane
// computes them with each thread running the reference's sequential sum
// (explicitly rounded multiply and add, no FMA contraction), which makes the
// result bit-identical to the CPU.  The nt+nx+ny-2 launches are captured once
// into a CUDA graph and replayed.
#include <sstream>

#include "internal.h"

namespace armab {
namespace {

constexpr int kThreads = 128;

__global__ void __launch_bounds__(kThreads)
ar64_plane_kernel(double* __restrict__ zeta, const double* __restrict__ phi,
                  int nt, int nx, int ny, int pt, int px, int py, int s, int t_lo) {
	const int t = t_lo + blockIdx.y;
	const int rem = s - t;                 // x + y
	const int x_lo = max(0, rem - (ny - 1));
	const int x = x_lo + blockIdx.x * kThreads + threadIdx.x;
	const int x_hi = min(nx - 1, rem);
	if (t >= nt || x > x_hi) return;
	const int y = rem - x;
	const long long sx = ny, st = (long long)nx * ny;
	const int m1 = min(t + 1, pt), m2 = min(x + 1, px), m3 = min(y + 1, py);
	double sum = 0.0;
	for (int k = 0; k < m1; ++k) {
		for (int i = 0; i < m2; ++i) {
			const double* prow = phi + (k * px + i) * py;
			const double* zrow = zeta + (t - k) * st + (x - i) * sx + y;
			for (int j = 0; j < m3; ++j)
				sum = __dadd_rn(sum, __dmul_rn(__ldg(prow + j), __ldg(zrow - j)));
		}
	}
	double* p = zeta + t * st + x * sx + y;
	*p = __dadd_rn(*p, sum);
}

}  // namespace

void launch_ar64(Ctx* c, const double* d_phi, const int order[3],
                 const int shape[3], double* d_zeta) {
	ProfScope prof_(c, "ar64");
	const int nt = shape[0], nx = shape[1], ny = shape[2];
	const int pt = order[0], px = order[1], py = order[2];
	if ((long long)nt * nx * ny == 0) return;
	std::ostringstream key;
	key << "ar64:" << (const void*)d_zeta << ':' << (const void*)d_phi << ':' << nt << ','
	    << nx << ',' << ny << ':' << pt << ',' << px << ',' << py;
	const int nplanes = nt + nx + ny - 2;
	auto it = c->graphs.find(key.str());
	if (it == c->graphs.end()) {
		cudaStream_t cap;
		ARMA_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
		cudaGraph_t graph;
		ARMA_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
		for (int s = 0; s < nplanes; ++s) {
			const int t_lo = max(0, s - (nx - 1) - (ny - 1));
			const int t_hi = min(nt - 1, s);
			const int nts = t_hi - t_lo + 1;
			const int xs = min(nx, s + 1);
			dim3 grid((xs + kThreads - 1) / kThreads, nts);
			ar64_plane_kernel<<<grid, kThreads, 0, cap>>>(d_zeta, d_phi, nt, nx, ny, pt, px,
			                                               py, s, t_lo);
		}
		ARMA_CUDA_TRY(cudaStreamEndCapture(cap, &graph));
		cudaGraphExec_t exec;
		ARMA_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
		ARMA_CUDA_TRY(cudaGraphDestroy(graph));
		ARMA_CUDA_TRY(cudaStreamDestroy(cap));
		it = c->graphs.emplace(key.str(), exec).first;
	}
	ARMA_CUDA_TRY(cudaGraphLaunch(it->second, c->stream));
	c->launches += uint64_t(nplanes);
}

}  // namespace armab
