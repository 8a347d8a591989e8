// Serving: device-resident AR surface streams generated chunk by chunk under
// continuous batching.
//
// A stream is an unbounded surface (t, x, y) of fixed nx x ny with one AR
// model and one dcmt stream; its chunk c holds slices [cT, (c+1)T).  The
// device keeps, per stream, two slice buffers of H + T slices (H = pt - 1).
// Chunk c is filtered in buffer c % 2 at slices [H, H+T), with the previous
// chunk's last H slices copied in front as a finished history, so every point
// sees exactly the neighbours it would see in one long surface.  The MT state
// is the raw window in front of the next unused word, rebuilt on the device
// from the tempered words the chunk consumed.  Chunk c is therefore the same,
// point for point, as slices [cT, (c+1)T) of a single surface generated in
// one call with the same seed; renormalisation (the reference's last-octant
// window rule) is fixed by the first chunk and applied to every output.
//
// Requests (the next chunk of a stream) are queued.  A host thread forms a
// batch from every queued request whose stream has no chunk in flight and
// whose state fits in the HBM budget, launches it on one of max_inflight CUDA
// streams (each with its own scratch arena), and completes the requests when
// the batch's event fires.  Batches on different CUDA streams overlap on the
// GPU, and requests that arrive while a batch runs join the next one.
//
// There is no counterpart of this layer in the reference; it reuses the
// reference-parity kernels (MT words, polar noise, FP32 compensated AR filter,
// variance window, linear velocity solver).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

using Clock = std::chrono::steady_clock;

constexpr int kCopyThreads = 256;
constexpr int kCopyBlocksPerJob = 64;
constexpr int kStreamLog2Seg = 16;  // MT segments of 2^16 words: short generation chains
constexpr int kMaxSlots = 8;

// ---------------------------------------------------------------- kernels
struct CopyJob {
	const float* src;
	float* dst;
	unsigned long long n;
	const double* scale;  // null: plain copy; else dst = fl32(src * scale) in FP64
};

__device__ __forceinline__ float scaled(float v, double s) { return float(double(v) * s); }

__global__ void __launch_bounds__(kCopyThreads) copy_batch_kernel(const CopyJob* __restrict__ jobs) {
	const CopyJob jb = jobs[blockIdx.x / kCopyBlocksPerJob];
	const int b = blockIdx.x % kCopyBlocksPerJob;
	const unsigned long long stride = (unsigned long long)kCopyBlocksPerJob * kCopyThreads;
	const unsigned long long first = (unsigned long long)b * kCopyThreads + threadIdx.x;
	const bool has_scale = jb.scale != nullptr;
	const double s = has_scale ? *jb.scale : 1.0;
	unsigned long long done = 0;
	if (((reinterpret_cast<uintptr_t>(jb.src) | reinterpret_cast<uintptr_t>(jb.dst)) & 15) == 0) {
		const unsigned long long n4 = jb.n / 4;
		const float4* s4 = reinterpret_cast<const float4*>(jb.src);
		float4* d4 = reinterpret_cast<float4*>(jb.dst);
		for (unsigned long long i = first; i < n4; i += stride) {
			float4 v = s4[i];
			if (has_scale) {
				v.x = scaled(v.x, s);
				v.y = scaled(v.y, s);
				v.z = scaled(v.z, s);
				v.w = scaled(v.w, s);
			}
			d4[i] = v;
		}
		done = n4 * 4;
	}
	for (unsigned long long i = done + first; i < jb.n; i += stride) {
		const float v = jb.src[i];
		jb.dst[i] = has_scale ? scaled(v, s) : v;
	}
}

void launch_copies(Ctx* c, const std::vector<CopyJob>& jobs) {
	if (jobs.empty()) return;
	ProfScope prof_(c, "copy");
	auto* d = static_cast<CopyJob*>(scratch_take(c, sizeof(CopyJob) * jobs.size()));
	ARMA_CUDA_TRY(cudaMemcpyAsync(d, jobs.data(), sizeof(CopyJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, c->stream));
	copy_batch_kernel<<<int(jobs.size()) * kCopyBlocksPerJob, kCopyThreads, 0, c->stream>>>(d);
	ARMA_CUDA_TRY(cudaGetLastError());
	c->launches += 1;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// ---------------------------------------------------------------- host state
struct StreamState {
	uint64_t id = 0;
	int nx = 0, ny = 0, pt = 0, px = 0, py = 0, H = 0;
	size_t n2 = 0;
	double var_wn = 0, acf0 = 0, delta[3] = {1, 1, 1};
	arma_mt_params mt{};
	uint32_t seed = 0;
	std::vector<float> coef;  // tile-kernel coefficient block
	// device state (one stream-ordered allocation)
	bool resident = false;
	char* mem = nullptr;
	size_t bytes = 0;
	float* buf[2] = {nullptr, nullptr};
	uint32_t* window[2] = {nullptr, nullptr};
	double* scale = nullptr;
	float* coef_d = nullptr;
	float* vel = nullptr;
	float* stage_z = nullptr;
	float* stage_v = nullptr;
	// progress
	uint64_t chunks_done = 0;
	bool busy = false;
	bool closed = false;
	int queued = 0;  // requests pending or in flight
};

struct Request {
	uint64_t id = 0, stream = 0;
	float* zeta_out = nullptr;
	float* vel_out = nullptr;
	bool zeta_dev = false, vel_dev = false;
	Clock::time_point submit, launch;
	double margin = 1.0;
	uint64_t chunk = 0;
	StreamState* st = nullptr;
};

struct Slot {
	arma_ctx* ctx = nullptr;
	cudaEvent_t begin = nullptr;  // batch start on the device
	cudaEvent_t done = nullptr;
	long long* h_pairs = nullptr;  // pinned: pairs per request, then the error word
	bool busy = false;
	std::vector<Request> reqs;
	bool failed = false;
	int fail_code = ARMA_OK;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
	return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace
}  // namespace armab

struct arma_server {
	int device = 0;
	arma_server_config cfg{};
	size_t budget = 0;
	std::mutex mu;
	std::condition_variable cv;       // work for the loop thread
	std::condition_variable cv_done;  // completions for pollers
	std::thread thread;
	bool stop = false;
	uint64_t next_stream = 1, next_request = 1;
	std::unordered_map<uint64_t, std::unique_ptr<armab::StreamState>> streams;
	std::deque<armab::Request> pending;
	std::deque<arma_completion> done;
	std::vector<armab::Slot> slots;
	arma_server_stats stats{};
	size_t resident_bytes = 0;
	// state blocks of closed streams kept for reuse by new streams of the
	// same footprint (allocating fresh device memory can take tens of ms)
	std::multimap<size_t, char*> spare;
	size_t spare_bytes = 0;
	std::string fatal;  // loop-thread failure outside any request

	void loop();
	void harvest();
	bool form_and_launch(armab::Slot& sl, std::unique_lock<std::mutex>& lk);
	uint64_t launch(armab::Slot& sl);
	void make_resident(armab::StreamState* st, armab::Ctx* c);
	void release(armab::StreamState* st, armab::Ctx* c);
	void reserve_block(armab::StreamState* st, armab::Ctx* c);
	size_t footprint(const armab::StreamState& st) const;
	void complete(armab::Slot& sl, size_t k, int status);
};

using namespace armab;

size_t arma_server::footprint(const StreamState& st) const {
	const size_t T = size_t(cfg.chunk_slices);
	const size_t nz = cfg.velocity ? size_t(cfg.nz) : 0;
	size_t b = 0;
	b += 2 * align256(sizeof(float) * (st.H + T) * st.n2);          // slice buffers
	b += 2 * align256(sizeof(uint32_t) * st.mt.nn);                 // MT windows
	b += align256(sizeof(double));                                  // scale
	b += align256(sizeof(float) * st.coef.size());                  // coefficients
	b += align256(sizeof(float) * T * nz * st.n2);                  // velocity
	b += align256(sizeof(float) * T * st.n2);                       // output staging
	b += align256(sizeof(float) * T * nz * st.n2);
	return b;
}

void arma_server::make_resident(StreamState* st, Ctx* c) {
	const size_t T = size_t(cfg.chunk_slices);
	const size_t nz = cfg.velocity ? size_t(cfg.nz) : 0;
	cudaStream_t s = c->stream;
	if (!st->mem) st->mem = static_cast<char*>(pool_alloc(c, st->bytes));
	char* m = st->mem;
	auto take = [&](size_t b) {
		char* r = m;
		m += align256(b);
		return r;
	};
	for (int k = 0; k < 2; ++k) st->buf[k] = reinterpret_cast<float*>(take(sizeof(float) * (st->H + T) * st->n2));
	for (int k = 0; k < 2; ++k) st->window[k] = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * st->mt.nn));
	st->scale = reinterpret_cast<double*>(take(sizeof(double)));
	st->coef_d = reinterpret_cast<float*>(take(sizeof(float) * st->coef.size()));
	st->vel = reinterpret_cast<float*>(take(sizeof(float) * T * nz * st->n2));
	st->stage_z = reinterpret_cast<float*>(take(sizeof(float) * T * st->n2));
	st->stage_v = reinterpret_cast<float*>(take(sizeof(float) * T * nz * st->n2));
	ARMA_CUDA_TRY(cudaMemcpyAsync(st->coef_d, st->coef.data(), sizeof(float) * st->coef.size(),
	                              cudaMemcpyHostToDevice, s));
	// the first chunk has no history: its filter reads none, its scale is
	// computed before use; a stream without renormalisation uses scale 1
	const double one = 1.0;
	ARMA_CUDA_TRY(cudaMemcpyAsync(st->scale, &one, sizeof(double), cudaMemcpyHostToDevice, s));
	st->resident = true;
}

void arma_server::release(StreamState* st, Ctx*) {
	if (st->resident && st->mem) {
		spare.emplace(st->bytes, st->mem);
		spare_bytes += st->bytes;
	}
	st->mem = nullptr;
	st->resident = false;
	resident_bytes -= st->bytes;
}

// A block for a stream being admitted: a spare one of the same size, else
// room is made in the budget by freeing spare blocks (the allocation itself
// happens in launch()).
void arma_server::reserve_block(StreamState* st, Ctx* c) {
	auto it = spare.find(st->bytes);
	if (it != spare.end()) {
		st->mem = it->second;
		spare_bytes -= it->first;
		spare.erase(it);
		return;
	}
	while (!spare.empty() && resident_bytes + spare_bytes > budget) {
		auto big = std::prev(spare.end());
		pool_free(c, big->second);
		spare_bytes -= big->first;
		spare.erase(big);
	}
}

// Requests are taken in arrival order; a request waits while its stream has a
// chunk in flight, and a stream's first request waits while its state does
// not fit in the budget next to the resident streams.
bool arma_server::form_and_launch(Slot& sl, std::unique_lock<std::mutex>& lk) {
	std::vector<Request> take;
	long long points = 0;
	const long long T = cfg.chunk_slices;
	for (auto it = pending.begin(); it != pending.end() && int(take.size()) < cfg.max_batch;) {
		StreamState* st = streams.at(it->stream).get();
		const long long np = T * (long long)st->n2;
		bool ok = !st->busy && (take.empty() || points + np <= cfg.max_batch_points);
		if (ok && !st->resident) {
			ok = resident_bytes + st->bytes <= budget;
			if (ok) {
				resident_bytes += st->bytes;  // reserved; allocated in launch()
				reserve_block(st, &sl.ctx->c);
			}
		}
		if (!ok) {
			++it;
			continue;
		}
		st->busy = true;
		it->st = st;
		it->chunk = st->chunks_done;
		take.push_back(*it);
		points += np;
		it = pending.erase(it);
	}
	if (take.empty()) return false;
	sl.reqs = std::move(take);
	sl.busy = true;
	sl.failed = false;
	const auto now = Clock::now();
	for (Request& r : sl.reqs) r.launch = now;
	lk.unlock();
	int code = ARMA_OK;
	std::string msg;
	uint64_t nl = 0;
	const auto t_launch = Clock::now();
	try {
		nl = launch(sl);
	} catch (const Error& e) {
		code = e.code;
		msg = e.msg;
	} catch (const std::exception& e) {
		code = ARMA_EINVAL;
		msg = e.what();
	}
	if (code != ARMA_OK) {
		cudaStreamSynchronize(sl.ctx->c.stream);
		cudaGetLastError();
		cudaEventRecord(sl.done, sl.ctx->c.stream);
	}
	lk.lock();
	if (code != ARMA_OK) {
		sl.failed = true;
		sl.fail_code = code;
		fatal = msg;
		for (Request& r : sl.reqs)  // reservations that were never made resident
			if (!r.st->resident) {
				resident_bytes -= r.st->bytes;
				if (r.st->mem) {
					spare.emplace(r.st->bytes, r.st->mem);
					spare_bytes += r.st->bytes;
					r.st->mem = nullptr;
				}
			}
	}
	stats.batches += 1;
	stats.launches += nl;
	const double lms = ms_between(t_launch, Clock::now());
	stats.launch_ms_total += lms;
	stats.launch_ms_max = std::max(stats.launch_ms_max, lms);
	return true;
}

uint64_t arma_server::launch(Slot& sl) {
	// host time per phase, reported on stderr for slow launches when the
	// ARMA_SERVE_TRACE environment variable is set
	static const bool trace = std::getenv("ARMA_SERVE_TRACE") != nullptr;
	double ph[10] = {0};
	auto tp = Clock::now();
	auto mark = [&](int k) {
		const auto now = Clock::now();
		ph[k] = ms_between(tp, now);
		tp = now;
	};
	Ctx* c = &sl.ctx->c;
	cudaStream_t s = c->stream;
	scratch_begin(c, 0);
	const int T = cfg.chunk_slices;
	const size_t n = sl.reqs.size();
	const int nz = cfg.velocity ? cfg.nz : 0;
	for (Request& r : sl.reqs)
		if (!r.st->resident) make_resident(r.st, c);
	const uint64_t launches0 = c->launches;
	ARMA_CUDA_TRY(cudaEventRecord(sl.begin, s));
	mark(0);
	// 1. history: the previous chunk's last H slices in front of this one
	std::vector<CopyJob> hist;
	for (Request& r : sl.reqs) {
		StreamState* st = r.st;
		const int cur = int(r.chunk & 1);
		if (r.chunk > 0 && st->H > 0)
			hist.push_back(CopyJob{st->buf[cur ^ 1] + size_t(T) * st->n2, st->buf[cur],
			                       size_t(st->H) * st->n2, nullptr});
	}
	launch_copies(c, hist);
	mark(1);
	// 2. MT words: from the seed (first chunk) or from the stream's window
	auto* d_att = static_cast<unsigned long long*>(scratch_take(c, sizeof(unsigned long long) * n));
	auto* d_pairs = static_cast<long long*>(scratch_take(c, sizeof(long long) * n));
	// a chunk whose noise runs short writes no attempt count: 0 marks it
	ARMA_CUDA_TRY(cudaMemsetAsync(d_att, 0, sizeof(unsigned long long) * n, s));
	std::vector<MtJob> mj(n);
	std::vector<uint64_t> att(n);
	for (size_t k = 0; k < n; ++k) {
		StreamState* st = sl.reqs[k].st;
		const size_t np = size_t(T) * st->n2;
		att[k] = noise_attempts(np, sl.reqs[k].margin * cfg.noise_margin);
		auto* w = static_cast<uint32_t*>(scratch_take(c, sizeof(uint32_t) * 4 * att[k]));
		const int cur = int(sl.reqs[k].chunk & 1);
		mj[k] = MtJob{st->mt, st->seed, 0, 4 * att[k], w,
		              sl.reqs[k].chunk > 0 ? st->window[cur] : nullptr};
	}
	launch_mt_generate_batch(c, mj, kStreamLog2Seg);
	mark(2);
	// 3. polar noise into the chunk slices, counting the attempts consumed
	std::vector<NoiseSpec> ns(n);
	for (size_t k = 0; k < n; ++k) {
		StreamState* st = sl.reqs[k].st;
		const int cur = int(sl.reqs[k].chunk & 1);
		ns[k] = NoiseSpec{mj[k].out, 4 * att[k], size_t(T) * st->n2, std::sqrt(st->var_wn),
		                  st->buf[cur] + size_t(st->H) * st->n2, d_att + k};
	}
	enqueue_white_noise_batch(c, ns, ARMA_FP32C, d_pairs);
	mark(3);
	// 4. the MT window for the next chunk
	std::vector<MtWindowSpec> ws(n);
	for (size_t k = 0; k < n; ++k) {
		StreamState* st = sl.reqs[k].st;
		const int cur = int(sl.reqs[k].chunk & 1);
		ws[k] = MtWindowSpec{st->mt, mj[k].out, 4 * att[k], d_att + k, st->window[cur ^ 1], nullptr};
	}
	launch_mt_window_update(c, ws);
	mark(4);
	// 5. the AR filter of every chunk in one launch
	const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
	std::vector<Ar32Surface> as(n);
	for (size_t k = 0; k < n; ++k) {
		StreamState* st = sl.reqs[k].st;
		const int cur = int(sl.reqs[k].chunk & 1);
		const size_t P = size_t(st->pt) * st->px * st->py;
		Ar32Surface& a = as[k];
		const bool first = sl.reqs[k].chunk == 0;
		a.nt = first ? T : st->H + T;
		a.nx = st->nx;
		a.ny = st->ny;
		a.pt = st->pt;
		a.px = st->px;
		a.py = st->py;
		a.zeta = first ? st->buf[cur] + size_t(st->H) * st->n2 : st->buf[cur];
		a.t0 = first ? 0 : st->H;
		a.phi = st->coef_d;
		a.phi_lo = st->coef_d + P;
		a.h = st->coef_d + 2 * P;
		a.tiles_x = (st->nx + tx - 1) / tx;
		a.tiles_y = (st->ny + ty - 1) / ty;
	}
	launch_ar32c(c, as, tx, ty, 0);
	mark(5);
	// 6. the stream's scale from its first chunk
	std::vector<RenormSpec> rs;
	for (Request& r : sl.reqs) {
		StreamState* st = r.st;
		if (r.chunk == 0 && st->acf0 > 0.0) {
			RenormSpec q;
			q.z = st->buf[int(r.chunk & 1)] + size_t(st->H) * st->n2;
			q.shape[0] = T;
			q.shape[1] = st->nx;
			q.shape[2] = st->ny;
			q.acf0 = st->acf0;
			q.d_scale = st->scale;
			rs.push_back(q);
		}
	}
	launch_renorm_batch(c, rs, ARMA_FP32C, false);
	mark(6);
	// 7. velocity potentials of the chunk slices: one set of launches per
	//    slice shape
	if (nz > 0) {
		std::map<std::pair<int, int>, std::vector<VelocitySurface>> groups;
		std::vector<std::vector<int>> tidx_keep;
		tidx_keep.reserve(sl.reqs.size());
		for (Request& r : sl.reqs) {
			StreamState* st = r.st;
			const int cur = int(r.chunk & 1);
			const bool first = r.chunk == 0;
			const int t0 = first ? 0 : st->H;
			tidx_keep.emplace_back(T);
			for (int t = 0; t < T; ++t) tidx_keep.back()[t] = t0 + t;
			VelocitySurface v;
			v.zeta = first ? st->buf[cur] + size_t(st->H) * st->n2 : st->buf[cur];
			v.out = st->vel;
			v.nt = t0 + T;
			v.t_idx = tidx_keep.back().data();
			v.ntd = T;
			v.dt = st->delta[0];
			groups[{st->nx, st->ny}].push_back(v);
		}
		for (auto& g : groups) {
			const ScratchMark mark = scratch_mark(c);  // groups run in order: share scratch
			launch_velocity_linear_batch(c, g.second.data(), int(g.second.size()), g.first.first,
			                             g.first.second, ARMA_FP32C, cfg.depth, cfg.z_levels, nz);
			scratch_release(c, mark);
		}
	}
	mark(7);
	// 8. outputs: scaled into the caller's device buffers or into staging
	std::vector<CopyJob> outs;
	for (Request& r : sl.reqs) {
		StreamState* st = r.st;
		const int cur = int(r.chunk & 1);
		const double* sc = st->acf0 > 0.0 ? st->scale : nullptr;
		const size_t nzeta = size_t(T) * st->n2;
		outs.push_back(CopyJob{st->buf[cur] + size_t(st->H) * st->n2,
		                       r.zeta_dev ? r.zeta_out : st->stage_z, nzeta, sc});
		if (nz > 0 && r.vel_out)
			outs.push_back(CopyJob{st->vel, r.vel_dev ? r.vel_out : st->stage_v, nzeta * nz, sc});
	}
	launch_copies(c, outs);
	for (Request& r : sl.reqs) {
		StreamState* st = r.st;
		const size_t nzeta = size_t(T) * st->n2;
		if (!r.zeta_dev)
			ARMA_CUDA_TRY(cudaMemcpyAsync(r.zeta_out, st->stage_z, sizeof(float) * nzeta,
			                              cudaMemcpyDeviceToHost, s));
		if (nz > 0 && r.vel_out && !r.vel_dev)
			ARMA_CUDA_TRY(cudaMemcpyAsync(r.vel_out, st->stage_v, sizeof(float) * nzeta * nz,
			                              cudaMemcpyDeviceToHost, s));
	}
	mark(8);
	// 9. status words back to pinned memory, then the completion event
	ARMA_CUDA_TRY(cudaMemcpyAsync(sl.h_pairs, d_pairs, sizeof(long long) * n, cudaMemcpyDeviceToHost, s));
	ARMA_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<int*>(sl.h_pairs + cfg.max_batch), c->d_err,
	                              sizeof(int), cudaMemcpyDeviceToHost, s));
	ARMA_CUDA_TRY(cudaEventRecord(sl.done, s));
	mark(9);
	if (trace) {
		double tot = 0;
		for (double v : ph) tot += v;
		if (tot > 5.0)
			std::fprintf(stderr,
			             "[arma serve] slow launch %.1f ms (%zu requests): resident %.1f hist %.1f "
			             "mt %.1f noise %.1f window %.1f ar %.1f renorm %.1f velocity %.1f out %.1f "
			             "status %.1f\n",
			             tot, n, ph[0], ph[1], ph[2], ph[3], ph[4], ph[5], ph[6], ph[7], ph[8], ph[9]);
	}
	return c->launches - launches0;
}

void arma_server::complete(Slot& sl, size_t k, int status) {
	Request& r = sl.reqs[k];
	StreamState* st = r.st;
	const auto now = Clock::now();
	arma_completion cpl{};
	cpl.request = r.id;
	cpl.stream = r.stream;
	cpl.chunk = r.chunk;
	cpl.status = status;
	cpl.latency_ms = ms_between(r.submit, now);
	cpl.queue_ms = ms_between(r.submit, r.launch);
	cpl.batch_size = int(sl.reqs.size());
	float dev_ms = 0.0f;
	if (!sl.failed && cudaEventElapsedTime(&dev_ms, sl.begin, sl.done) == cudaSuccess)
		cpl.device_ms = dev_ms;
	else
		cudaGetLastError();
	done.push_back(cpl);
	st->busy = false;
	st->queued -= 1;
	if (status == ARMA_OK) {
		st->chunks_done += 1;
		stats.points += uint64_t(cfg.chunk_slices) * st->n2;
	}
	stats.completed += 1;
}

// Completes every slot whose batch has finished.  A request whose noise ran
// short of accepted polar attempts (rare by construction) is queued again at
// the front with more attempts; the stream's buffers and MT window of the
// previous chunk are untouched, so the redo is exact.
void arma_server::harvest() {
	bool any = false;
	for (Slot& sl : slots) {
		if (!sl.busy) continue;
		const cudaError_t q = cudaEventQuery(sl.done);
		if (q == cudaErrorNotReady) continue;
		any = true;
		int batch_status = ARMA_OK;
		if (q != cudaSuccess) {
			cudaGetLastError();
			batch_status = ARMA_ECUDA;
			fatal = cudaGetErrorString(q);
		} else if (sl.failed) {
			batch_status = sl.fail_code;
		} else {
			const int err = *reinterpret_cast<const int*>(sl.h_pairs + cfg.max_batch);
			if (err != DEV_OK) {
				batch_status = err == DEV_TIMEOUT ? ARMA_ETIMEDOUT : ARMA_ECUDA;
				fatal = "a bounded device wait gave up";
				cudaMemsetAsync(sl.ctx->c.d_err, 0, sizeof(int), sl.ctx->c.stream);
			}
		}
		std::vector<Request> redo;
		for (size_t k = 0; k < sl.reqs.size(); ++k) {
			Request& r = sl.reqs[k];
			if (batch_status == ARMA_OK) {
				const long long need = (long long)cfg.chunk_slices * (long long)r.st->n2 / 2;
				if (sl.h_pairs[k] < need) {
					r.margin *= 1.5;
					r.st->busy = false;
					redo.push_back(r);
					stats.redone += 1;
					continue;
				}
			}
			complete(sl, k, batch_status);
		}
		for (auto it = redo.rbegin(); it != redo.rend(); ++it) pending.push_front(*it);
		sl.reqs.clear();
		sl.busy = false;
	}
	// closed streams with nothing queued give their memory back
	for (auto it = streams.begin(); it != streams.end();) {
		StreamState* st = it->second.get();
		if (st->closed && st->queued == 0 && !st->busy) {
			if (st->resident) release(st, &slots[0].ctx->c);
			it = streams.erase(it);
			any = true;
		} else {
			++it;
		}
	}
	if (any) cv_done.notify_all();
}

void arma_server::loop() {
	cudaSetDevice(device);
	std::unique_lock<std::mutex> lk(mu);
	for (;;) {
		harvest();
		bool launched = false;
		for (Slot& sl : slots) {
			if (sl.busy) continue;
			if (!form_and_launch(sl, lk)) break;
			launched = true;
		}
		bool inflight = false;
		for (Slot& sl : slots) inflight = inflight || sl.busy;
		if (stop && !inflight && pending.empty()) break;
		if (inflight || launched) {
			cv.wait_for(lk, std::chrono::microseconds(20));
		} else {
			cv.wait(lk);
		}
	}
	cv_done.notify_all();
}

extern "C" {

int arma_server_config_default(arma_server_config* cfg) {
	if (!cfg) return ARMA_EINVAL;
	*cfg = arma_server_config{};
	cfg->chunk_slices = 64;
	cfg->max_inflight = 3;
	cfg->max_batch = 64;
	cfg->max_batch_points = 1ll << 26;
	cfg->hbm_budget = 0;
	cfg->velocity = 1;
	cfg->depth = INFINITY;
	cfg->nz = 1;
	cfg->z_levels[0] = 0.0;
	cfg->noise_margin = 1.0;
	return ARMA_OK;
}

int arma_server_create(int device, const arma_server_config* cfg, arma_server** out) {
	return guard([&] {
		ARMA_REQUIRE(cfg && out, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(cfg->chunk_slices >= 2 && cfg->chunk_slices % 2 == 0, ARMA_EINVAL,
		             "chunk_slices must be even and >= 2");
		ARMA_REQUIRE(cfg->max_inflight >= 1 && cfg->max_inflight <= kMaxSlots, ARMA_EINVAL,
		             "max_inflight must be in [1, 8]");
		ARMA_REQUIRE(cfg->max_batch >= 1 && cfg->max_batch_points >= 1, ARMA_EINVAL,
		             "bad batch limits");
		ARMA_REQUIRE(!cfg->velocity || (cfg->nz >= 1 && cfg->nz <= 8), ARMA_EINVAL,
		             "velocity needs 1..8 z levels");
		ARMA_REQUIRE(!cfg->velocity || cfg->depth > 0, ARMA_EINVAL, "depth must be positive");
		ARMA_REQUIRE(cfg->noise_margin > 0, ARMA_EINVAL, "noise_margin must be positive");
		std::unique_ptr<arma_server> srv(new arma_server());
		srv->device = device;
		srv->cfg = *cfg;
		ARMA_CUDA_TRY(cudaSetDevice(device));
		size_t free_b = 0, total_b = 0;
		ARMA_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
		srv->budget = cfg->hbm_budget ? cfg->hbm_budget : free_b / 2;
		srv->slots.resize(cfg->max_inflight);
		for (Slot& sl : srv->slots) {
			const int rc = arma_ctx_create(device, &sl.ctx);
			if (rc != ARMA_OK) throw Error{rc, last_error()};
			sl.ctx->c.profiling = cfg->profile != 0;
			// scratch of a full batch, reserved up front: MT words (~10.2 bytes
			// a point), spectra for several depths, velocity work buffers
			const size_t per_point = 11 + (cfg->velocity && cfg->nz > 1 ? 8 * size_t(cfg->nz) : 0);
			scratch_reserve(&sl.ctx->c, size_t(cfg->max_batch_points) * per_point + (640u << 20));
			ARMA_CUDA_TRY(cudaEventCreate(&sl.begin));
			ARMA_CUDA_TRY(cudaEventCreate(&sl.done));
			ARMA_CUDA_TRY(cudaHostAlloc(&sl.h_pairs, sizeof(long long) * (cfg->max_batch + 1),
			                            cudaHostAllocDefault));
		}
		// back the library pool with physical memory for stream state now, so
		// that admitting a stream does not wait for the driver to map memory
		{
			Ctx* c0 = &srv->slots[0].ctx->c;
			const size_t warm = std::min(srv->budget, size_t(4) << 30);
			void* p = pool_alloc(c0, warm);
			pool_free(c0, p);
			ARMA_CUDA_TRY(cudaStreamSynchronize(c0->stream));
		}
		arma_server* raw = srv.get();
		srv->thread = std::thread([raw] { raw->loop(); });
		*out = srv.release();
	});
}

int arma_server_destroy(arma_server* srv) {
	return guard([&] {
		if (!srv) return;
		{
			std::lock_guard<std::mutex> lk(srv->mu);
			srv->stop = true;
			for (auto& kv : srv->streams) kv.second->closed = true;
		}
		srv->cv.notify_all();
		if (srv->thread.joinable()) srv->thread.join();
		cudaSetDevice(srv->device);
		for (auto& kv : srv->streams)
			if (kv.second->resident) srv->release(kv.second.get(), &srv->slots[0].ctx->c);
		for (auto& kv : srv->spare) pool_free(&srv->slots[0].ctx->c, kv.second);
		srv->spare.clear();
		for (Slot& sl : srv->slots) {
			if (sl.ctx) cudaStreamSynchronize(sl.ctx->c.stream);
			if (sl.begin) cudaEventDestroy(sl.begin);
			if (sl.done) cudaEventDestroy(sl.done);
			if (sl.h_pairs) cudaFreeHost(sl.h_pairs);
			if (sl.ctx) arma_ctx_destroy(sl.ctx);
		}
		delete srv;
	});
}

int arma_stream_open(arma_server* srv, const arma_stream_spec* spec, uint64_t* stream_id) {
	return guard([&] {
		ARMA_REQUIRE(srv && spec && stream_id && spec->phi, ARMA_EINVAL, "null argument");
		require_mt(&spec->mt);
		const int* o = spec->order;
		ARMA_REQUIRE(spec->nx > 0 && spec->ny > 0 && o[0] > 0 && o[1] > 0 && o[2] > 0, ARMA_EINVAL,
		             "Bad \"stream\": dimensions must be positive");
		ARMA_REQUIRE(o[1] <= ar32c_tile_x() + 1 && o[2] <= 13 && o[0] * o[1] <= ar32c_max_tap_rows(),
		             ARMA_ENOTSUP, "AR order not supported by the FP32 tile kernel");
		ARMA_REQUIRE(o[0] - 1 <= srv->cfg.chunk_slices, ARMA_EINVAL,
		             "a chunk must be at least as long as the AR history (order t - 1)");
		ARMA_REQUIRE(spec->var_wn >= 0.0 && std::isfinite(spec->var_wn), ARMA_EINVAL,
		             "variance is less than zero");
		ARMA_REQUIRE((long long)srv->cfg.chunk_slices * spec->nx * spec->ny % 2 == 0, ARMA_EINVAL,
		             "chunk point count must be even");
		if (srv->cfg.velocity)
			ARMA_REQUIRE(velocity_supported(spec->nx, spec->ny), ARMA_ENOTSUP,
			             "velocity solver: slice sides must be in [4, 1024] with prime factors <= 64");
		std::unique_ptr<StreamState> st(new StreamState());
		st->nx = spec->nx;
		st->ny = spec->ny;
		st->pt = o[0];
		st->px = o[1];
		st->py = o[2];
		st->H = o[0] - 1;
		st->n2 = size_t(spec->nx) * spec->ny;
		st->var_wn = spec->var_wn;
		st->acf0 = spec->acf0;
		for (int i = 0; i < 3; ++i) st->delta[i] = spec->delta[i] > 0 ? spec->delta[i] : 1.0;
		st->mt = spec->mt;
		st->seed = spec->seed;
		st->coef.resize(ar32_coefficient_count(o));
		ar32_coefficients(spec->phi, o, st->coef.data());
		st->bytes = srv->footprint(*st);
		ARMA_REQUIRE(st->bytes <= srv->budget, ARMA_ENOMEM,
		             "stream state is larger than the server's HBM budget");
		std::lock_guard<std::mutex> lk(srv->mu);
		st->id = srv->next_stream++;
		*stream_id = st->id;
		srv->streams.emplace(st->id, std::move(st));
	});
}

int arma_stream_close(arma_server* srv, uint64_t stream_id) {
	return guard([&] {
		ARMA_REQUIRE(srv, ARMA_EINVAL, "null argument");
		{
			std::lock_guard<std::mutex> lk(srv->mu);
			auto it = srv->streams.find(stream_id);
			ARMA_REQUIRE(it != srv->streams.end() && !it->second->closed, ARMA_EINVAL,
			             "unknown stream");
			it->second->closed = true;
		}
		srv->cv.notify_all();
	});
}

int arma_stream_submit(arma_server* srv, uint64_t stream_id, float* zeta_out, float* velocity_out,
                       uint64_t* request_id) {
	return guard([&] {
		ARMA_REQUIRE(srv && zeta_out, ARMA_EINVAL, "null argument");
		Request r;
		r.stream = stream_id;
		r.zeta_out = zeta_out;
		r.vel_out = srv->cfg.velocity ? velocity_out : nullptr;
		// outputs must be device memory or page-locked host memory: a copy to
		// pageable memory would block the serving thread
		auto kind = [](const void* p, bool* dev) {
			cudaPointerAttributes a{};
			if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
				cudaGetLastError();
				throw Error{ARMA_EINVAL, "cannot classify an output pointer"};
			}
			ARMA_REQUIRE(a.type != cudaMemoryTypeUnregistered, ARMA_EINVAL,
			             "outputs must be device memory or page-locked host memory");
			*dev = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
		};
		ARMA_CUDA_TRY(cudaSetDevice(srv->device));
		kind(zeta_out, &r.zeta_dev);
		if (r.vel_out) kind(r.vel_out, &r.vel_dev);
		{
			std::lock_guard<std::mutex> lk(srv->mu);
			auto it = srv->streams.find(stream_id);
			ARMA_REQUIRE(it != srv->streams.end() && !it->second->closed, ARMA_EINVAL,
			             "unknown stream");
			r.id = srv->next_request++;
			r.submit = Clock::now();
			it->second->queued += 1;
			srv->pending.push_back(r);
			srv->stats.submitted += 1;
			if (request_id) *request_id = r.id;
		}
		srv->cv.notify_all();
	});
}

int arma_server_poll(arma_server* srv, arma_completion* out, int max, int timeout_ms, int* n) {
	return guard([&] {
		ARMA_REQUIRE(srv && out && n && max > 0, ARMA_EINVAL, "null argument");
		std::unique_lock<std::mutex> lk(srv->mu);
		if (srv->done.empty() && timeout_ms != 0) {
			auto ready = [&] { return !srv->done.empty() || srv->stop; };
			if (timeout_ms < 0)
				srv->cv_done.wait(lk, ready);
			else
				srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
		}
		int k = 0;
		while (k < max && !srv->done.empty()) {
			out[k++] = srv->done.front();
			srv->done.pop_front();
		}
		*n = k;
	});
}

int arma_server_stats_get(arma_server* srv, arma_server_stats* out) {
	return guard([&] {
		ARMA_REQUIRE(srv && out, ARMA_EINVAL, "null argument");
		std::lock_guard<std::mutex> lk(srv->mu);
		*out = srv->stats;
		out->resident_bytes = srv->resident_bytes;
		out->budget_bytes = srv->budget;
		out->streams = int(srv->streams.size());
		int res = 0, infl = 0;
		for (auto& kv : srv->streams) res += kv.second->resident ? 1 : 0;
		for (const Slot& sl : srv->slots) infl += sl.busy ? 1 : 0;
		out->resident_streams = res;
		out->inflight = infl;
		out->pending = int(srv->pending.size());
	});
}

int arma_server_profile(arma_server* srv, const char* name, double* ms, uint64_t* launches) {
	return guard([&] {
		ARMA_REQUIRE(srv && name && ms && launches, ARMA_EINVAL, "null argument");
		std::lock_guard<std::mutex> lk(srv->mu);
		*ms = 0.0;
		*launches = 0;
		ARMA_CUDA_TRY(cudaSetDevice(srv->device));
		for (Slot& sl : srv->slots) {
			if (sl.busy) continue;  // its events may not have fired yet
			resolve_profile(&sl.ctx->c);
			auto it = sl.ctx->c.prof_ms.find(name);
			if (it != sl.ctx->c.prof_ms.end()) {
				*ms += it->second;
				*launches += uint64_t(sl.ctx->c.prof_count[name]);
			}
		}
	});
}

int arma_server_last_failure(arma_server* srv, char* buf, size_t len) {
	if (!srv || !buf || len == 0) return ARMA_EINVAL;
	std::lock_guard<std::mutex> lk(srv->mu);
	std::snprintf(buf, len, "%s", srv->fatal.c_str());
	return ARMA_OK;
}

}  // extern "C"
