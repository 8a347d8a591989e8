// C ABI: argument checking, error mapping, context and scratch management,
// and the orchestration of the device kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "distributions.h"
#include "internal.h"

namespace armab {

namespace {
thread_local std::string g_last_error;

arma_ctx* outer(Ctx* c) {
	return reinterpret_cast<arma_ctx*>(reinterpret_cast<char*>(c) - offsetof(arma_ctx, c));
}

void require_shape(const int s[3], const char* name) {
	ARMA_REQUIRE(s && s[0] > 0 && s[1] > 0 && s[2] > 0, ARMA_EINVAL,
	             std::string("Bad \"") + name + "\": dimensions must be positive");
}

size_t elem_size(int precision) {
	ARMA_REQUIRE(precision == ARMA_FP64 || precision == ARMA_FP32C, ARMA_EINVAL,
	             "bad precision");
	return precision == ARMA_FP64 ? sizeof(double) : sizeof(float);
}

}  // namespace

// Host-side copy of sgenrand-independent validation of a parameter set.
// A parameter set is used only if its recurrence and tempering are well
// formed: besides sizing the generator, the tempering shifts must lie in
// [1, 31] (the device inverts the tempering by fixed-point iteration, which
// advances by the shift).
void require_mt(const arma_mt_params* p) {
	ARMA_REQUIRE(p, ARMA_EINVAL, "null MT parameter set");
	auto shift_ok = [](int s) { return s >= 1 && s <= 31; };
	ARMA_REQUIRE(p->ww == 32 && p->nn > 1 && p->mm > 0 && p->mm < p->nn && p->rr >= 0 &&
	                 p->rr < 32 && shift_ok(p->shift0) && shift_ok(p->shift1) &&
	                 shift_ok(p->shiftB) && shift_ok(p->shiftC),
	             ARMA_EINVAL, "bad MT parameter set");
}

uint64_t noise_attempts(size_t n, double margin) {
	const double pairs = std::ceil(n / 2.0);
	return uint64_t((pairs * (4.0 / dist::kPi) + 8.0 * std::sqrt(pairs) + 256.0) * margin);
}

namespace {

void white_noise(Ctx* c, const arma_mt_params& p, uint32_t seed, double stddev, size_t n,
                 int precision, void* d_out) {
	ARMA_REQUIRE(stddev >= 0.0 && std::isfinite(stddev), ARMA_EINVAL,
	             "variance is less than zero");
	if (n == 0) return;
	double margin = 1.0;
	for (int round = 0; round < 8; ++round) {
		const uint64_t n_att = noise_attempts(n, margin);
		uint32_t* words = static_cast<uint32_t*>(scratch_take(c, sizeof(uint32_t) * 4 * n_att));
		launch_mt_generate(c, p, seed, 0, 4 * n_att, words);
		if (launch_white_noise(c, words, 4 * n_att, stddev, n, precision, d_out)) return;
		margin *= 1.5;
	}
	throw Error{ARMA_ECUDA, "white noise: rejection sampling did not converge"};
}

// White noise for many surfaces: all MT streams in a few launches, the polar
// transforms in one.  The plan holds every surface's MT job (its words in
// scratch); noise_enqueue generates the words and the normal values of the
// surfaces idx and returns the device array of their accepted pairs (in idx
// order).
struct NoisePlan {
	std::vector<MtJob> jobs;
	std::vector<uint64_t> att;
};

NoisePlan noise_plan(Ctx* c, const arma_surface* s, int n) {
	NoisePlan plan;
	plan.jobs.resize(n);
	plan.att.resize(n);
	for (int k = 0; k < n; ++k) {
		ARMA_REQUIRE(s[k].var_wn >= 0.0 && std::isfinite(s[k].var_wn), ARMA_EINVAL,
		             "variance is less than zero");
		const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
		plan.att[k] = noise_attempts(np, c->noise_margin);
		plan.jobs[k] = MtJob{s[k].mt, s[k].seed, 0, 4 * plan.att[k],
		                     static_cast<uint32_t*>(scratch_take(c, sizeof(uint32_t) * 4 * plan.att[k]))};
	}
	return plan;
}

// words_ready: the surfaces' MT words were generated already (one wide launch
// for a whole batch); only the polar transform is enqueued.
long long* noise_enqueue(Ctx* c, const arma_surface* s, const NoisePlan& plan,
                         const std::vector<int>& idx, int precision, const std::vector<void*>& dz,
                         bool words_ready = false) {
	const int n = int(idx.size());
	long long* d_pairs = static_cast<long long*>(scratch_take(c, sizeof(long long) * n));
	if (!words_ready) {
		std::vector<MtJob> jobs(n);
		for (int q = 0; q < n; ++q) jobs[q] = plan.jobs[idx[q]];
		launch_mt_generate_batch(c, jobs, c->tuning.mt_log2_segment);
	}
	std::vector<NoiseSpec> specs(n);
	for (int q = 0; q < n; ++q) {
		const int k = idx[q];
		const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
		specs[q] = NoiseSpec{plan.jobs[k].out, 4 * plan.att[k], np, std::sqrt(s[k].var_wn), dz[k]};
	}
	enqueue_white_noise_batch(c, specs, precision, d_pairs);
	return d_pairs;
}

long long* white_noise_batch_enqueue(Ctx* c, const arma_surface* s, int n, int precision,
                                     const std::vector<void*>& dz) {
	const NoisePlan plan = noise_plan(c, s, n);
	std::vector<int> idx(n);
	for (int k = 0; k < n; ++k) idx[k] = k;
	return noise_enqueue(c, s, plan, idx, precision, dz);
}

// True when surface k's accepted pairs do not cover its points (rare: the
// attempts carry an 8 sigma margin).
bool noise_short(const arma_surface& s, long long pairs) {
	const size_t np = size_t(s.shape[0]) * s.shape[1] * s.shape[2];
	return uint64_t(pairs) * 2 < np;
}

void white_noise_batch(Ctx* c, const arma_surface* s, int n, int precision,
                       const std::vector<void*>& dz) {
	long long* d_pairs = white_noise_batch_enqueue(c, s, n, precision, dz);
	std::vector<long long> pairs(n);
	ARMA_CUDA_TRY(copy_async(c, pairs.data(), d_pairs, sizeof(long long) * n,
	                              cudaMemcpyDeviceToHost, c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	check_device_error(c);
	for (int k = 0; k < n; ++k) {
		const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
		if (noise_short(s[k], pairs[k]))  // the sequential generator instead
			white_noise(c, s[k].mt, s[k].seed, std::sqrt(s[k].var_wn), np, precision, dz[k]);
	}
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

cudaMemPool_t library_pool(int device) {
	static std::mutex m;
	static std::map<int, cudaMemPool_t> pools;
	std::lock_guard<std::mutex> lk(m);
	auto it = pools.find(device);
	if (it != pools.end()) return it->second;
	cudaMemPoolProps props{};
	props.allocType = cudaMemAllocationTypePinned;
	props.location.type = cudaMemLocationTypeDevice;
	props.location.id = device;
	cudaMemPool_t pool;
	ARMA_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
	uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool for reuse
	ARMA_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
	// never make an allocation on one stream wait for a free still queued on
	// another (concurrent serving batches would serialise); reuse only
	// blocks whose free has completed, else grow the pool
	int no = 0;
	ARMA_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
	pools.emplace(device, pool);
	return pool;
}

void* pool_alloc(Ctx* c, size_t bytes) {
	void* p = nullptr;
	if (cudaMallocFromPoolAsync(&p, bytes, library_pool(c->device), c->stream) != cudaSuccess) {
		cudaGetLastError();
		throw Error{ARMA_ENOMEM, "device allocation failed"};
	}
	return p;
}

void pool_free(Ctx* c, void* p) {
	if (p) cudaFreeAsync(p, c->stream);
}

// Chunks come from the library's stream-ordered pool, so growing or merging
// the arena never synchronises the device.
void scratch_begin(Ctx* c, size_t) {
	arma_ctx* o = outer(c);
	if (o->chunks.size() > 1 || (o->chunks.size() == 1 && o->chunks[0].second < o->high_water)) {
		for (auto& ch : o->chunks) pool_free(c, ch.first);
		o->chunks.clear();
		char* p = static_cast<char*>(pool_alloc(c, o->high_water));
		o->chunks.emplace_back(p, o->high_water);
	}
	o->used = 0;
	o->taken = 0;
}

void* scratch_take(Ctx* c, size_t bytes) {
	arma_ctx* o = outer(c);
	bytes = (bytes + 255) & ~size_t(255);
	if (o->chunks.empty() || o->used + bytes > o->chunks.back().second) {
		const size_t sz = std::max(bytes, size_t(64) << 20);
		char* p = static_cast<char*>(pool_alloc(c, sz));
		o->chunks.emplace_back(p, sz);
		o->used = 0;
	}
	void* r = o->chunks.back().first + o->used;
	o->used += bytes;
	o->taken += bytes;
	o->high_water = std::max(o->high_water, o->taken);
	return r;
}

void scratch_reserve(Ctx* c, size_t bytes) {
	arma_ctx* o = outer(c);
	o->high_water = std::max(o->high_water, bytes);
	scratch_begin(c, 0);
	if (o->chunks.empty()) {
		char* p = static_cast<char*>(pool_alloc(c, o->high_water));
		o->chunks.emplace_back(p, o->high_water);
	}
}

ScratchMark scratch_mark(Ctx* c) {
	arma_ctx* o = outer(c);
	return ScratchMark{o->chunks.size(), o->used, o->taken};
}

void scratch_release(Ctx* c, const ScratchMark& m) {
	arma_ctx* o = outer(c);
	if (o->chunks.size() != m.chunks) return;  // grew meanwhile: keep going forward
	o->used = m.used;
	o->taken = m.taken;
}

ProfScope::ProfScope(Ctx* c, const char* name) : c_(c) {
	if (!c->profiling) return;
	Ctx::Pending p;
	p.name = name;
	ARMA_CUDA_TRY(cudaEventCreate(&p.start));
	ARMA_CUDA_TRY(cudaEventCreate(&p.stop));
	ARMA_CUDA_TRY(cudaEventRecord(p.start, c->stream));
	c->pending.push_back(p);
	idx_ = int(c->pending.size()) - 1;
}

ProfScope::~ProfScope() {
	if (idx_ >= 0) cudaEventRecord(c_->pending[idx_].stop, c_->stream);
}

void resolve_profile(Ctx* c) {
	if (c->pending.empty()) return;
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	for (auto& p : c->pending) {
		float ms = 0.0f;
		ARMA_CUDA_TRY(cudaEventElapsedTime(&ms, p.start, p.stop));
		c->prof_ms[p.name] += ms;
		c->prof_count[p.name] += 1;
		cudaEventDestroy(p.start);
		cudaEventDestroy(p.stop);
	}
	c->pending.clear();
}

void check_device_error(Ctx* c) {
	int h = 0;
	ARMA_CUDA_TRY(copy_async(c, &h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (h == DEV_TIMEOUT) {
		ARMA_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
		throw Error{ARMA_ETIMEDOUT,
		            "a bounded device wait gave up (a tile dependency or a noise block's "
		            "predecessor count never arrived)"};
	}
	if (h != DEV_OK) {
		ARMA_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
		throw Error{ARMA_ECUDA, "device-side check failed"};
	}
}

}  // namespace armab

using namespace armab;

extern "C" {

int arma_version(void) { return ARMA_B200_VERSION; }

int arma_last_error(char* buf, size_t len) {
	if (!buf || len == 0) return ARMA_EINVAL;
	std::snprintf(buf, len, "%s", g_last_error.c_str());
	return ARMA_OK;
}

int arma_ctx_create(int device, arma_ctx** out) {
	return guard([&] {
		ARMA_REQUIRE(out, ARMA_EINVAL, "null output pointer");
		int ndev = 0;
		ARMA_CUDA_TRY(cudaGetDeviceCount(&ndev));
		ARMA_REQUIRE(device >= 0 && device < ndev, ARMA_EINVAL, "bad device index");
		ARMA_CUDA_TRY(cudaSetDevice(device));
		std::unique_ptr<arma_ctx> ctx(new arma_ctx());
		ctx->c.device = device;
		ARMA_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
		ctx->c.own_stream = true;
		ARMA_CUDA_TRY(cudaMalloc(&ctx->c.d_err, sizeof(int)));
		ARMA_CUDA_TRY(cudaMemset(ctx->c.d_err, 0, sizeof(int)));
		ARMA_CUDA_TRY(cudaDeviceGetAttribute(&ctx->c.num_sms, cudaDevAttrMultiProcessorCount, device));
		*out = ctx.release();
	});
}

int arma_ctx_destroy(arma_ctx* ctx) {
	return guard([&] {
		if (!ctx) return;
		cudaSetDevice(ctx->c.device);
		cudaStreamSynchronize(ctx->c.stream);
		for (auto& p : ctx->c.pending) {
			cudaEventDestroy(p.start);
			cudaEventDestroy(p.stop);
		}
		for (auto& kv : ctx->c.graphs) cudaGraphExecDestroy(kv.second);
		for (auto& kv : ctx->c.nit_tables) cudaFree(kv.second);
		for (auto& ch : ctx->chunks) pool_free(&ctx->c, ch.first);
		cudaStreamSynchronize(ctx->c.stream);
		if (ctx->c.side_stream) {
			cudaStreamSynchronize(ctx->c.side_stream);
			cudaStreamDestroy(ctx->c.side_stream);
		}
		if (ctx->c.copy_stream) {
			cudaStreamSynchronize(ctx->c.copy_stream);
			cudaStreamDestroy(ctx->c.copy_stream);
		}
		cudaFree(ctx->c.d_err);
		if (ctx->c.own_stream) cudaStreamDestroy(ctx->c.stream);
		delete ctx;
	});
}

int arma_ctx_set_stream(arma_ctx* ctx, void* stream) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		// scratch allocated in the old stream's order must be complete before
		// the new stream uses it
		ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
		if (ctx->c.own_stream) ARMA_CUDA_TRY(cudaStreamDestroy(ctx->c.stream));
		ctx->c.stream = static_cast<cudaStream_t>(stream);
		ctx->c.own_stream = false;
	});
}

int arma_ctx_synchronize(arma_ctx* ctx) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
	});
}

int arma_ctx_launch_count(arma_ctx* ctx, uint64_t* count) {
	return guard([&] {
		ARMA_REQUIRE(ctx && count, ARMA_EINVAL, "null argument");
		*count = ctx->c.launches;
	});
}

int arma_ctx_transfer_bytes(arma_ctx* ctx, uint64_t* h2d, uint64_t* d2h) {
	return guard([&] {
		ARMA_REQUIRE(ctx && h2d && d2h, ARMA_EINVAL, "null argument");
		*h2d = ctx->c.h2d_bytes;
		*d2h = ctx->c.d2h_bytes;
	});
}

int arma_ctx_set_profiling(arma_ctx* ctx, int enabled) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		ctx->c.profiling = enabled != 0;
	});
}

int arma_ctx_set_noise_margin(arma_ctx* ctx, double margin) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		ARMA_REQUIRE(margin > 0.0 && std::isfinite(margin), ARMA_EINVAL,
		             "noise margin must be positive");
		ctx->c.noise_margin = margin;
	});
}

namespace {
void require_tuning(const arma_tuning* t) {
	ARMA_REQUIRE(t, ARMA_EINVAL, "null tuning");
	ARMA_REQUIRE(t->mt_log2_segment >= 16 && t->mt_log2_segment <= 22, ARMA_EINVAL,
	             "mt_log2_segment must be in [16, 22]");
	ARMA_REQUIRE(t->ar_ctas_per_sm >= 0 && t->ar_ctas_per_sm <= 32, ARMA_EINVAL,
	             "ar_ctas_per_sm must be in [0, 32]");
	ARMA_REQUIRE(t->host_groups >= 1 && t->host_groups <= 16, ARMA_EINVAL,
	             "host_groups must be in [1, 16]");
	ARMA_REQUIRE(t->host_first > 0.0 && t->host_first < 1.0, ARMA_EINVAL,
	             "host_first must be in (0, 1)");
}
}  // namespace

int arma_ctx_get_tuning(arma_ctx* ctx, arma_tuning* out) {
	return guard([&] {
		ARMA_REQUIRE(ctx && out, ARMA_EINVAL, "null argument");
		*out = ctx->c.tuning;
	});
}

int arma_ctx_set_tuning(arma_ctx* ctx, const arma_tuning* t) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		require_tuning(t);
		ctx->c.tuning = *t;
	});
}

int arma_ctx_profile(arma_ctx* ctx, const char* name, double* ms, uint64_t* launches) {
	return guard([&] {
		ARMA_REQUIRE(ctx && name && ms && launches, ARMA_EINVAL, "null argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		resolve_profile(&ctx->c);
		auto it = ctx->c.prof_ms.find(name);
		*ms = it == ctx->c.prof_ms.end() ? 0.0 : it->second;
		auto jt = ctx->c.prof_count.find(name);
		*launches = jt == ctx->c.prof_count.end() ? 0 : uint64_t(jt->second);
	});
}

int arma_ctx_profile_reset(arma_ctx* ctx) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null context");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		resolve_profile(&ctx->c);
		ctx->c.prof_ms.clear();
		ctx->c.prof_count.clear();
	});
}

// ---------------------------------------------------------------- MT sets
int arma_mt19937_params(arma_mt_params* p) {
	return guard([&] {
		ARMA_REQUIRE(p, ARMA_EINVAL, "null output pointer");
		std::memset(p, 0, sizeof(*p));
		p->aaa = 0x9908b0dfu;
		p->mm = 397;
		p->nn = 624;
		p->rr = 31;
		p->ww = 32;
		p->wmask = 0xffffffffu;
		p->umask = 0x80000000u;
		p->lmask = 0x7fffffffu;
		p->shift0 = 11;
		p->shift1 = 18;
		p->shiftB = 7;
		p->shiftC = 15;
		p->maskB = 0x9d2c5680u;
		p->maskC = 0xefc60000u;
		p->i = 624;
	});
}

int arma_mt_create(int w, int p, int id, uint32_t seed, arma_mt_params* out) {
	return guard([&] {
		ARMA_REQUIRE(out, ARMA_EINVAL, "null output pointer");
		ARMA_REQUIRE(w == 32, ARMA_EINVAL, "only w = 32 parameter sets are supported");
		ARMA_REQUIRE(dcmt::mersenne_exponent(p), ARMA_EINVAL,
		             "p must be a Mersenne exponent between 521 and 44497");
		ARMA_REQUIRE(id >= 0 && id < 65536, ARMA_EINVAL, "id must be in [0, 65536)");
		arma_mt_params r;
		if (dcmt::create(p, id, seed, &r) != 0)
			throw Error{ARMA_ENUMERIC, "bad MT: no primitive characteristic polynomial for id " +
			                               std::to_string(id)};
		*out = r;
	});
}

int arma_mt_is_primitive(const arma_mt_params* p, int* primitive) {
	return guard([&] {
		ARMA_REQUIRE(primitive, ARMA_EINVAL, "null output pointer");
		require_mt(p);
		*primitive = dcmt::mersenne_exponent(32 * p->nn - p->rr) && dcmt::is_primitive(*p) ? 1 : 0;
	});
}

int arma_mt_equidistribution(const arma_mt_params* p, int vmax, int* k_out) {
	return guard([&] {
		ARMA_REQUIRE(k_out && vmax >= 1 && vmax <= 32, ARMA_EINVAL, "bad argument");
		require_mt(p);
		for (int v = 1; v <= vmax; ++v) k_out[v - 1] = int(dcmt::equidistribution(*p, v));
	});
}

namespace {
constexpr size_t kMtRecord = 72;  // raw x86-64 mt_struct incl. padding + pointer

bool read_record(std::ifstream& in, arma_mt_params* p) {
	unsigned char hdr[kMtRecord];
	if (!in.read(reinterpret_cast<char*>(hdr), kMtRecord)) return false;
	std::memcpy(p, hdr, sizeof(arma_mt_params));
	if (p->nn <= 0 || p->nn > (1 << 20)) throw Error{ARMA_EIO, "malformed MT configuration file"};
	in.seekg(std::streamoff(p->nn) * 4, std::ios::cur);
	return bool(in);
}
}  // namespace

int arma_mt_file_count(const char* path, int* count) {
	return guard([&] {
		ARMA_REQUIRE(path && count, ARMA_EINVAL, "null argument");
		std::ifstream in(path, std::ios::binary);
		if (!in)
			throw Error{ARMA_EIO,
			            std::string("Mersenne Twister configuration file not found: ") + path};
		int n = 0;
		arma_mt_params p;
		while (read_record(in, &p)) ++n;
		*count = n;
	});
}

int arma_mt_file_read(const char* path, int index, arma_mt_params* out) {
	return guard([&] {
		ARMA_REQUIRE(path && out && index >= 0, ARMA_EINVAL, "bad argument");
		std::ifstream in(path, std::ios::binary);
		if (!in)
			throw Error{ARMA_EIO,
			            std::string("Mersenne Twister configuration file not found: ") + path};
		arma_mt_params p;
		for (int k = 0; k <= index; ++k)
			if (!read_record(in, &p))
				throw Error{ARMA_EPRNG, "bad number of MT configs"};
		*out = p;
	});
}

int arma_mt_file_write(const char* path, const arma_mt_params* sets, int n) {
	return guard([&] {
		ARMA_REQUIRE(path && sets && n > 0, ARMA_EINVAL, "bad argument");
		std::ofstream out(path, std::ios::binary);
		ARMA_REQUIRE(bool(out), ARMA_EIO, std::string("cannot write ") + path);
		for (int k = 0; k < n; ++k) {
			require_mt(&sets[k]);
			unsigned char hdr[kMtRecord] = {0};
			std::memcpy(hdr, &sets[k], sizeof(arma_mt_params));
			out.write(reinterpret_cast<const char*>(hdr), kMtRecord);
			// state words: sgenrand_mt(0), which read_parallel_mts replaces anyway
			uint32_t s = 0;
			for (int i = 0; i < sets[k].nn; ++i) {
				const uint32_t w = s & sets[k].wmask;
				out.write(reinterpret_cast<const char*>(&w), 4);
				s = 1812433253u * (s ^ (s >> 30)) + uint32_t(i + 1);
			}
		}
		ARMA_REQUIRE(bool(out), ARMA_EIO, std::string("cannot write ") + path);
	});
}

int arma_mt_genrand(arma_ctx* ctx, const arma_mt_params* p, uint32_t seed, uint64_t offset,
                    size_t n, uint32_t* d_out) {
	return guard([&] {
		ARMA_REQUIRE(ctx && d_out, ARMA_EINVAL, "null argument");
		require_mt(p);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_mt_generate(&ctx->c, *p, seed, offset, n, d_out);
	});
}

// ---------------------------------------------------------------- fit
int arma_auto_covariance(const double* in, const int shape[3], double* out) {
	return guard([&] {
		ARMA_REQUIRE(in && out && shape, ARMA_EINVAL, "null argument");
		require_shape(shape, "array");
		const size_t n = size_t(shape[0]) * shape[1] * shape[2];
		const std::vector<double> r = auto_covariance(std::vector<double>(in, in + n), shape);
		std::copy(r.begin(), r.end(), out);
	});
}

int arma_auto_covariance_device(arma_ctx* ctx, const void* d_in, const int shape[3],
                                int precision, double* d_out) {
	return guard([&] {
		ARMA_REQUIRE(ctx && d_in && shape && d_out, ARMA_EINVAL, "null argument");
		require_shape(shape, "array");
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_auto_covariance(&ctx->c, d_in, shape, precision, d_out);
	});
}

int arma_acf_eval(int kind, double amplitude, double velocity, const double alpha[3],
                  const double beta[2], const double delta[3], const int shape[3],
                  double* acf) {
	return guard([&] {
		ARMA_REQUIRE(alpha && beta && delta && acf, ARMA_EINVAL, "null argument");
		require_shape(shape, "acf");
		ARMA_REQUIRE(kind == ARMA_ACF_STANDING || kind == ARMA_ACF_PROPAGATING, ARMA_EINVAL,
		             "bad ACF function");
		acf_eval(kind, amplitude, velocity, alpha, beta, delta, shape, acf);
	});
}

int arma_ar_fit(const double* acf, const int acf_shape[3], const int order[3], int method,
                double* phi, double* var_wn) {
	return guard([&] {
		ARMA_REQUIRE(acf && phi && var_wn, ARMA_EINVAL, "null argument");
		require_shape(acf_shape, "acf");
		require_shape(order, "order");
		ARMA_REQUIRE(order[0] <= acf_shape[0] && order[1] <= acf_shape[1] &&
		                 order[2] <= acf_shape[2],
		             ARMA_EINVAL, "bad AR model order");
		const int info = fit_gauss_table(acf, acf_shape, order, method, phi, var_wn);
		ARMA_REQUIRE(info == 0, ARMA_ENUMERIC,
		             "Yule-Walker matrix is not positive definite (pivot " +
		                 std::to_string(info) + ")");
	});
}

int arma_ar_fit_analytic(int kind, double amplitude, double velocity, const double alpha[3],
                         const double beta[2], const double delta[3], const int order[3],
                         double* phi, double* var_wn) {
	return guard([&] {
		ARMA_REQUIRE(alpha && beta && delta && phi && var_wn, ARMA_EINVAL, "null argument");
		require_shape(order, "order");
		const int info =
		    fit_analytic(kind, amplitude, velocity, alpha, beta, delta, order, phi, var_wn);
		ARMA_REQUIRE(info == 0, ARMA_ENUMERIC,
		             "Yule-Walker matrix is not positive definite (pivot " +
		                 std::to_string(info) + ")");
	});
}

// ---------------------------------------------------------------- noise, AR
int arma_white_noise(arma_ctx* ctx, const arma_mt_params* p, uint32_t seed, double stddev,
                     size_t n, int precision, void* d_out) {
	return guard([&] {
		ARMA_REQUIRE(ctx && d_out, ARMA_EINVAL, "null argument");
		require_mt(p);
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		white_noise(&ctx->c, *p, seed, stddev, n, precision, d_out);
	});
}

}  // extern "C"

namespace armab {

size_t ar32_coefficient_count(const int order[3]) {
	return 2 * size_t(order[0]) * order[1] * order[2] + size_t(ar32c_tile_x()) * ar32c_tile_y();
}

void ar32_coefficients(const double* phi, const int order[3], float* b) {
	const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
	const size_t nh = size_t(tx) * ty;
	const int P = order[0] * order[1] * order[2];
	std::vector<double> h(nh);
	intra_slice_response(phi, order, tx, ty, h.data());
	for (int i = 0; i < P; ++i) {
		b[i] = float(phi[i]);
		b[P + i] = float(phi[i] - double(b[i]));
	}
	// The lo parts correct the rounding of phi to float; their effect on the
	// surface is concentrated in few (k, i) tap rows.  Rows are kept in
	// decreasing order of their lo energy until the dropped rows hold at most
	// 1e-4 of it (1 % of the norm); the others are zeroed and the filter skips
	// their second FMA chain.  On the configured models this keeps 33-94 % of
	// the rows and adds at most ~1e-6 RMS to the FP32 surface error.
	{
		const int rows = order[0] * order[1], py = order[2];
		std::vector<std::pair<double, int>> e(rows);
		double total = 0.0;
		for (int r = 0; r < rows; ++r) {
			double v = 0.0;
			for (int j = 0; j < py; ++j) v += double(b[P + r * py + j]) * b[P + r * py + j];
			e[r] = {v, r};
			total += v;
		}
		std::sort(e.begin(), e.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
		double kept = 0.0;
		for (const auto& [v, r] : e) {
			if (total - kept <= 1e-4 * total) {
				for (int j = 0; j < py; ++j) b[P + r * py + j] = 0.0f;
			} else {
				kept += v;
			}
		}
	}
	for (size_t i = 0; i < nh; ++i) b[2 * P + i] = float(h[i]);
}

}  // namespace armab

extern "C" {

namespace {

// Device copies of the hi/lo float split of phi and of the intra-slice
// response H for the FP32 tile kernel, for n surfaces in one upload.
std::vector<Ar32Surface> ar32_surfaces(Ctx* c, int n, const double* const* phis,
                                       const int* const* orders, const int* const* shapes,
                                       float* const* zetas) {
	const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
	std::vector<size_t> off(n + 1, 0);
	for (int k = 0; k < n; ++k) off[k + 1] = off[k] + ar32_coefficient_count(orders[k]);
	std::vector<float> buf(off[n]);
	// independent per surface (FP64 H and the lo-row selection): one thread each
#pragma omp parallel for schedule(dynamic, 4) if (n >= 8)
	for (int k = 0; k < n; ++k) ar32_coefficients(phis[k], orders[k], buf.data() + off[k]);
	float* d = static_cast<float*>(scratch_take(c, sizeof(float) * buf.size()));
	ARMA_CUDA_TRY(copy_async(c, d, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice,
	                              c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));  // buf is pageable and local
	std::vector<Ar32Surface> out(n);
	for (int k = 0; k < n; ++k) {
		const int P = orders[k][0] * orders[k][1] * orders[k][2];
		float* dk = d + off[k];
		Ar32Surface& s = out[k];
		s.nt = shapes[k][0];
		s.nx = shapes[k][1];
		s.ny = shapes[k][2];
		s.pt = orders[k][0];
		s.px = orders[k][1];
		s.py = orders[k][2];
		s.zeta = zetas[k];
		s.phi = dk;
		s.phi_lo = dk + P;
		s.h = dk + 2 * P;
		s.tiles_x = (s.nx + tx - 1) / tx;
		s.tiles_y = (s.ny + ty - 1) / ty;
	}
	return out;
}

void ar_filter(Ctx* c, const double* phi, const int order[3], const int shape[3],
               int precision, void* d_zeta) {
	const int P = order[0] * order[1] * order[2];
	if (precision == ARMA_FP64) {
		double* d_phi = static_cast<double*>(scratch_take(c, sizeof(double) * P));
		ARMA_CUDA_TRY(copy_async(c, d_phi, phi, sizeof(double) * P, cudaMemcpyHostToDevice,
		                              c->stream));
		launch_ar64(c, d_phi, order, shape, static_cast<double*>(d_zeta));
	} else {
		const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
		float* z = static_cast<float*>(d_zeta);
		std::vector<Ar32Surface> s = ar32_surfaces(c, 1, &phi, &order, &shape, &z);
		launch_ar32c(c, s, tx, ty, 1);
		check_device_error(c);
	}
}

void require_order(const int order[3]) {
	require_shape(order, "order");
	ARMA_REQUIRE(order[0] <= 16 && order[1] <= 16 && order[2] <= 16, ARMA_ENOTSUP,
	             "AR order above 16 per dimension is not supported on the device");
}

}  // namespace

int arma_ar_filter(arma_ctx* ctx, const double* phi, const int order[3], const int shape[3],
                   int precision, void* d_zeta) {
	return guard([&] {
		ARMA_REQUIRE(ctx && phi && d_zeta, ARMA_EINVAL, "null argument");
		require_shape(shape, "out_grid");
		require_order(order);
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		ar_filter(&ctx->c, phi, order, shape, precision, d_zeta);
	});
}

int arma_ar_filter_strip(arma_ctx* ctx, const double* phi, const int order[3], const int shape[3],
                         int t0, int given_rows, float* d_zeta) {
	return guard([&] {
		ARMA_REQUIRE(ctx && phi && d_zeta, ARMA_EINVAL, "null argument");
		require_shape(shape, "out_grid");
		require_order(order);
		const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
		ARMA_REQUIRE(t0 >= 0 && t0 < shape[0], ARMA_EINVAL, "t0 must be in [0, nt)");
		ARMA_REQUIRE(given_rows >= 0 && given_rows % tx == 0 && given_rows < shape[1], ARMA_EINVAL,
		             "given_rows must be a multiple of 16 rows below nx");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		float* z = d_zeta;
		std::vector<Ar32Surface> s = ar32_surfaces(&ctx->c, 1, &phi, &order, &shape, &z);
		s[0].t0 = t0;
		s[0].given_tx = given_rows / tx;
		launch_ar32c(&ctx->c, s, tx, ty, 1);
		check_device_error(&ctx->c);
	});
}

int arma_variance_renorm(arma_ctx* ctx, void* d_zeta, const int shape[3], int precision,
                         double acf0, double* scale_out) {
	return guard([&] {
		ARMA_REQUIRE(ctx && d_zeta, ARMA_EINVAL, "null argument");
		require_shape(shape, "out_grid");
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		double* d_scale = static_cast<double*>(scratch_take(&ctx->c, sizeof(double)));
		launch_renorm(&ctx->c, d_zeta, shape, precision, acf0, d_scale);
		double s = 0.0;
		ARMA_CUDA_TRY(copy_async(&ctx->c, &s, d_scale, sizeof(double), cudaMemcpyDeviceToHost,
		                              ctx->c.stream));
		ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
		if (scale_out) *scale_out = s;
	});
}

int arma_nit_apply(arma_ctx* ctx, int d, const double params[3], double stdev, int method,
                   const double interval[2], double eps, int max_iter, int lut_nodes,
                   double lut_range, size_t n, int precision, void* d_zeta) {
	return guard([&] {
		ARMA_REQUIRE(ctx && params && d_zeta, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(d == ARMA_NIT_GRAM_CHARLIER || d == ARMA_NIT_SKEW_NORMAL, ARMA_EINVAL,
		             "bad distribution");
		ARMA_REQUIRE(stdev > 0.0, ARMA_EINVAL, "bad stdev");
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		if (method == ARMA_NIT_BISECTION) {
			ARMA_REQUIRE(interval && max_iter > 0 && eps > 0.0, ARMA_EINVAL, "bad cdf_solver");
			launch_nit_bisection(&ctx->c, d, params, stdev, interval[0], interval[1], eps,
			                     max_iter, n, precision, d_zeta);
		} else {
			ARMA_REQUIRE(lut_nodes >= 4 && lut_range > 0.0, ARMA_EINVAL, "bad NIT table");
			double x0, dx;
			std::vector<double> y;
			nit_build_lut(d, params, stdev, lut_nodes, lut_range, &x0, &dx, y);
			const std::vector<double> coef = nit_lut_coefficients(y);
			const std::vector<float> coef_f(coef.begin(), coef.end());
			const bool fp64 = precision == ARMA_FP64;
			const size_t bytes = fp64 ? sizeof(double) * coef.size() : sizeof(float) * coef.size();
			void* d_lut = scratch_take(&ctx->c, bytes);
			ARMA_CUDA_TRY(copy_async(&ctx->c, d_lut,
			                         fp64 ? static_cast<const void*>(coef.data()) : coef_f.data(),
			                         bytes, cudaMemcpyHostToDevice, ctx->c.stream));
			launch_nit_lut(&ctx->c, d_lut, lut_nodes, x0, dx, n, precision, d_zeta);
			ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
		}
	});
}

namespace {
int velocity_call(arma_ctx* ctx, const void* d_zeta, const int shape[3], int precision,
                  const double delta[3], double depth, const double* z, int nz, const int* t_idx,
                  int ntd, void* d_phi_out, int mode) {
	return guard([&] {
		ARMA_REQUIRE(ctx && d_zeta && delta && z && t_idx && d_phi_out, ARMA_EINVAL,
		             "null argument");
		require_shape(shape, "out_grid");
		ARMA_REQUIRE(nz > 0 && ntd > 0, ARMA_EINVAL, "Bad \"domain\": empty");
		for (int i = 0; i < ntd; ++i)
			ARMA_REQUIRE(t_idx[i] >= 0 && t_idx[i] < shape[0], ARMA_EINVAL,
			             "Bad \"domain\": t outside the surface");
		for (int j = 0; j < nz; ++j)
			ARMA_REQUIRE(!(z[j] < -depth), ARMA_EINVAL, "min(z) is less than -h");
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_velocity_linear(&ctx->c, d_zeta, shape, precision, delta, depth, z, nz, t_idx,
		                       ntd, d_phi_out, mode);
		ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
	});
}
}  // namespace

int arma_velocity_linear(arma_ctx* ctx, const void* d_zeta, const int shape[3], int precision,
                         const double delta[3], double depth, const double* z, int nz,
                         const int* t_idx, int ntd, void* d_phi_out) {
	return velocity_call(ctx, d_zeta, shape, precision, delta, depth, z, nz, t_idx, ntd, d_phi_out,
	                     0);
}

int arma_velocity_high_amplitude(arma_ctx* ctx, const void* d_zeta, const int shape[3],
                                 int precision, const double delta[3], double depth,
                                 const double* z, int nz, const int* t_idx, int ntd,
                                 void* d_phi_out) {
	return velocity_call(ctx, d_zeta, shape, precision, delta, depth, z, nz, t_idx, ntd, d_phi_out,
	                     1);
}

int arma_velocity_linear_batch(arma_ctx* ctx, const arma_velocity_job* jobs, int n, int nx, int ny,
                               int precision, double depth, const double* z, int nz) {
	return guard([&] {
		ARMA_REQUIRE(ctx && jobs && z && n >= 0, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(nx > 0 && ny > 0 && nz > 0, ARMA_EINVAL, "Bad \"domain\": empty");
		for (int j = 0; j < nz; ++j)
			ARMA_REQUIRE(!(z[j] < -depth), ARMA_EINVAL, "min(z) is less than -h");
		elem_size(precision);
		std::vector<VelocitySurface> v(n);
		for (int k = 0; k < n; ++k) {
			const arma_velocity_job& j = jobs[k];
			ARMA_REQUIRE(j.d_zeta && j.d_out && j.t_idx && j.nt > 0 && j.ntd > 0, ARMA_EINVAL,
			             "bad velocity job");
			for (int i = 0; i < j.ntd; ++i)
				ARMA_REQUIRE(j.t_idx[i] >= 0 && j.t_idx[i] < j.nt, ARMA_EINVAL,
				             "Bad \"domain\": t outside the surface");
			v[k] = VelocitySurface{j.d_zeta, j.d_out, j.nt, j.t_idx, j.ntd, j.dt > 0 ? j.dt : 1.0};
		}
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_velocity_linear_batch(&ctx->c, v.data(), n, nx, ny, precision, depth, z, nz);
		ARMA_CUDA_TRY(cudaStreamSynchronize(ctx->c.stream));
	});
}

// ---------------------------------------------------------------- batches
namespace {

// A surface's NIT table for the fused renormalisation pass (p == nullptr: none).
struct SurfaceLut {
	const void* p = nullptr;
	int nodes = 0;
	double x0 = 0.0, inv_dx = 0.0;
};

void renorm_surfaces(Ctx* c, arma_surface* s, int n, int precision, const std::vector<void*>& dz,
                     bool host, const SurfaceLut* luts);
void pipelined_host_output(Ctx* c, arma_surface* s, int n, const std::vector<void*>& dz,
                           const SurfaceLut* luts);

RenormSpec renorm_spec(const arma_surface& s, void* z, double* d_scale, const SurfaceLut* lut) {
	RenormSpec r{z, {s.shape[0], s.shape[1], s.shape[2]}, s.acf0, d_scale};
	if (lut && lut->p) {
		r.lut = lut->p;
		r.lut_nodes = lut->nodes;
		r.lut_x0 = lut->x0;
		r.lut_inv_dx = lut->inv_dx;
	}
	return r;
}

// redo: the noise's accepted-pair counts are read back before the filter
// (white_noise_batch, with its sequential fallback); otherwise the FP32 path
// enqueues the noise, builds the filter's coefficient tables on the host while
// the device generates it, and checks the counts at the end, generating a
// surface whose noise ran short again on its own.
void batch(Ctx* c, arma_surface* s, int n, int precision, bool host, bool redo = false,
           const SurfaceLut* luts = nullptr) {
	const size_t es = elem_size(precision);
	std::vector<void*> dz(n);
	for (int k = 0; k < n; ++k) {
		require_shape(s[k].shape, "out_grid");
		require_order(s[k].order);
		require_mt(&s[k].mt);
		ARMA_REQUIRE(s[k].phi && s[k].d_zeta, ARMA_EINVAL, "null surface buffer");
		ARMA_REQUIRE(s[k].var_wn >= 0.0, ARMA_EINVAL, "variance is less than zero");
		const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
		dz[k] = host ? scratch_take(c, np * es) : s[k].d_zeta;
	}
	if (host && precision == ARMA_FP32C && n >= 4 && !redo) {
		pipelined_host_output(c, s, n, dz, luts);
		return;
	}
	if (precision == ARMA_FP64) {
		white_noise_batch(c, s, n, precision, dz);
		for (int k = 0; k < n; ++k) ar_filter(c, s[k].phi, s[k].order, s[k].shape, precision, dz[k]);
		renorm_surfaces(c, s, n, precision, dz, host, luts);
		return;
	}
	long long* d_pairs = nullptr;
	if (redo) white_noise_batch(c, s, n, precision, dz);
	else d_pairs = white_noise_batch_enqueue(c, s, n, precision, dz);
	const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
	std::vector<const double*> phis(n);
	std::vector<const int*> ords(n), shps(n);
	std::vector<float*> zs(n);
	for (int k = 0; k < n; ++k) {
		phis[k] = s[k].phi;
		ords[k] = s[k].order;
		shps[k] = s[k].shape;
		zs[k] = static_cast<float*>(dz[k]);
	}
	std::vector<Ar32Surface> as =
	    ar32_surfaces(c, n, phis.data(), ords.data(), shps.data(), zs.data());
	launch_ar32c(c, as, tx, ty, 1);
	std::vector<long long> pairs(n, 0);
	if (d_pairs)
		ARMA_CUDA_TRY(copy_async(c, pairs.data(), d_pairs, sizeof(long long) * n,
		                              cudaMemcpyDeviceToHost, c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	check_device_error(c);
	renorm_surfaces(c, s, n, precision, dz, host, luts);
	if (d_pairs)
		for (int k = 0; k < n; ++k)
			if (noise_short(s[k], pairs[k]))
				batch(c, &s[k], 1, precision, host, true, luts ? luts + k : nullptr);
}

// FP32 surfaces into host buffers with the device->host copies overlapped with
// the computation.  The surfaces are ordered by the length of their filter's
// dependency chain (slices + tile rows + tile columns) and cut, in that order,
// into groups holding shares of the total points x taps (a first share, then
// equal ones), so that each group's persistent filter launch ends without a
// long tail and the first group, of the shortest chains, is ready early.  The
// groups' white noise, filter and renormalisation alternate between two
// compute streams, so that one group's launches fill the SMs that the other's
// tail leaves idle; each group's device->host copies run on a copy stream as
// soon as its renormalisation is done.  The copies bound the call: the
// computation outpaces the PCIe link after the first group.
void pipelined_host_output(Ctx* c, arma_surface* s, int n, const std::vector<void*>& dz,
                           const SurfaceLut* luts) {
	const int G = std::min(std::max(c->tuning.host_groups, 1), std::max(n, 1));
	std::vector<double> frac(G, G > 1 ? (1.0 - c->tuning.host_first) / (G - 1) : 1.0);
	if (G > 1) frac[0] = c->tuning.host_first;
	const int tx = ar32c_tile_x(), ty = ar32c_tile_y();
	std::vector<double> work(n);
	double total = 0.0;
	for (int k = 0; k < n; ++k) {
		work[k] = double(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2] * s[k].order[0] *
		          s[k].order[1] * s[k].order[2];
		total += work[k];
	}
	// shortest dependency chains first, cut into consecutive groups by share
	auto chain = [&](int k) {
		return s[k].shape[0] + (s[k].shape[1] + tx - 1) / tx + (s[k].shape[2] + ty - 1) / ty;
	};
	std::vector<int> order(n);
	for (int k = 0; k < n; ++k) order[k] = k;
	std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
		return chain(a) != chain(b) ? chain(a) < chain(b) : work[a] < work[b];
	});
	std::vector<std::vector<int>> members(G);
	{
		int g = 0;
		double bound = frac[0] * total, acc = 0.0;
		for (int k : order) {
			while (g + 1 < G && acc >= bound) bound += frac[++g] * total;
			members[g].push_back(k);
			acc += work[k];
		}
	}
	// the filter's coefficient tables of every surface (host work, one
	// upload), built while the device generates the first group's noise
	std::vector<const double*> phis(n);
	std::vector<const int*> ords(n), shps(n);
	std::vector<float*> zs(n);
	for (int k = 0; k < n; ++k) {
		phis[k] = s[k].phi;
		ords[k] = s[k].order;
		shps[k] = s[k].shape;
		zs[k] = static_cast<float*>(dz[k]);
	}
	std::vector<Ar32Surface> as;
	// Each group's noise is enqueued without reading its accepted-pair counts
	// back (a device->host read on the context's stream would queue behind the
	// previous groups' copies); the counts are checked at the end.
	std::vector<long long*> d_pairs(G, nullptr);
	// every surface's MT jump-ahead windows and then all its words once, in
	// wide launches (per group they would be narrow, latency-bound trees and
	// short generation launches); the groups run only the polar transform
	NoisePlan plan = noise_plan(c, s, n);
	auto noise = [&](int g) {
		d_pairs[g] = noise_enqueue(c, s, plan, members[g], ARMA_FP32C, dz, true);
	};
	if (!c->copy_stream)
		ARMA_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
	if (!c->side_stream)
		ARMA_CUDA_TRY(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
	double* d_scale = static_cast<double*>(scratch_take(c, sizeof(double) * n));
	std::vector<cudaEvent_t> ev;
	auto event = [&](cudaStream_t st) {
		cudaEvent_t e;
		ARMA_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		ev.push_back(e);
		ARMA_CUDA_TRY(cudaEventRecord(e, st));
		return e;
	};
	const cudaStream_t main_stream = c->stream;
	auto release = [&] {
		c->stream = main_stream;
		for (cudaEvent_t e : ev) cudaEventDestroy(e);
	};
	try {
		launch_mt_prepare(c, plan.jobs, c->tuning.mt_log2_segment);
		launch_mt_generate_batch(c, plan.jobs, c->tuning.mt_log2_segment);
		// the side stream starts after the caller's earlier work and the words
		ARMA_CUDA_TRY(cudaStreamWaitEvent(c->side_stream, event(main_stream), 0));
		for (int g = 0; g < G; ++g) {
			if (members[g].empty()) continue;
			// the context's launch helpers enqueue on c->stream
			c->stream = (g % 2 == 0) ? main_stream : c->side_stream;
			noise(g);
			if (as.empty()) {
				as = ar32_surfaces(c, n, phis.data(), ords.data(), shps.data(), zs.data());
				// the coefficient tables' upload precedes the other stream's filters
				const cudaStream_t other = c->stream == main_stream ? c->side_stream : main_stream;
				ARMA_CUDA_TRY(cudaStreamWaitEvent(other, event(c->stream), 0));
			}
			std::vector<Ar32Surface> ga;
			std::vector<RenormSpec> rs;
			for (int k : members[g]) {
				ga.push_back(as[k]);
				if (s[k].acf0 > 0.0)
					rs.push_back(renorm_spec(s[k], dz[k], d_scale + k, luts ? luts + k : nullptr));
			}
			launch_ar32c(c, ga, tx, ty, 1);
			launch_renorm_batch(c, rs, ARMA_FP32C);
			ARMA_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, event(c->stream), 0));
			for (int k : members[g]) {
				const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
				ARMA_CUDA_TRY(copy_async(c, s[k].d_zeta, dz[k], np * sizeof(float),
				                              cudaMemcpyDeviceToHost, c->copy_stream));
			}
		}
		c->stream = main_stream;
		ARMA_CUDA_TRY(cudaStreamWaitEvent(main_stream, event(c->side_stream), 0));
		std::vector<double> sc(n, 1.0);
		ARMA_CUDA_TRY(copy_async(c, sc.data(), d_scale, sizeof(double) * n, cudaMemcpyDeviceToHost,
		                              c->stream));
		ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
		ARMA_CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
		check_device_error(c);
		for (int k = 0; k < n; ++k) s[k].scale = s[k].acf0 > 0.0 ? sc[k] : 1.0;
		// a surface whose noise ran short is generated again on its own
		for (int g = 0; g < G; ++g) {
			if (members[g].empty()) continue;
			std::vector<long long> pairs(members[g].size());
			ARMA_CUDA_TRY(cudaMemcpy(pairs.data(), d_pairs[g], sizeof(long long) * pairs.size(),
			                         cudaMemcpyDeviceToHost));
			for (size_t q = 0; q < pairs.size(); ++q)
				if (noise_short(s[members[g][q]], pairs[q]))
					batch(c, &s[members[g][q]], 1, ARMA_FP32C, true, true,
					      luts ? luts + members[g][q] : nullptr);
		}
	} catch (...) {
		cudaStreamSynchronize(c->side_stream);
		cudaStreamSynchronize(c->copy_stream);
		release();
		throw;
	}
	release();
}

// The variance renormalisation of each surface with acf0 > 0 (and the copy to
// the host buffers when `host`), then the scales back into s[k].scale.
void renorm_surfaces(Ctx* c, arma_surface* s, int n, int precision, const std::vector<void*>& dz,
                     bool host, const SurfaceLut* luts) {
	const size_t es = elem_size(precision);
	double* d_scale = static_cast<double*>(scratch_take(c, sizeof(double) * n));
	std::vector<RenormSpec> rs;
	for (int k = 0; k < n; ++k)
		if (s[k].acf0 > 0.0) rs.push_back(renorm_spec(s[k], dz[k], d_scale + k, luts ? luts + k : nullptr));
	launch_renorm_batch(c, rs, precision);
	if (host) {
		for (int k = 0; k < n; ++k) {
			const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
			ARMA_CUDA_TRY(copy_async(c, s[k].d_zeta, dz[k], np * es, cudaMemcpyDeviceToHost,
			                              c->stream));
		}
	}
	std::vector<double> sc(n, 1.0);
	ARMA_CUDA_TRY(copy_async(c, sc.data(), d_scale, sizeof(double) * n, cudaMemcpyDeviceToHost,
	                              c->stream));
	ARMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
	for (int k = 0; k < n; ++k) s[k].scale = s[k].acf0 > 0.0 ? sc[k] : 1.0;
}

// White noise into scratch, the MA filter into each surface's buffer, then the
// renormalisation (MA_model::do_generate, src/generator/ma_model.cc:30-40).
void ma_batch(Ctx* c, arma_surface* s, int n, int precision) {
	const size_t es = elem_size(precision);
	std::vector<void*> eps(n), dz(n);
	for (int k = 0; k < n; ++k) {
		require_shape(s[k].shape, "out_grid");
		require_shape(s[k].order, "order");
		require_mt(&s[k].mt);
		ARMA_REQUIRE(s[k].phi && s[k].d_zeta, ARMA_EINVAL, "null surface buffer");
		ARMA_REQUIRE(s[k].var_wn >= 0.0, ARMA_EINVAL, "variance is less than zero");
		const size_t np = size_t(s[k].shape[0]) * s[k].shape[1] * s[k].shape[2];
		eps[k] = scratch_take(c, np * es);
		dz[k] = s[k].d_zeta;
	}
	white_noise_batch(c, s, n, precision, eps);
	for (int k = 0; k < n; ++k)
		launch_ma_filter(c, s[k].phi, s[k].order, s[k].shape, precision, eps[k], dz[k]);
	renorm_surfaces(c, s, n, precision, dz, false, nullptr);
}

}  // namespace

}  // extern "C"

namespace armab {
void batch_generate_device(Ctx* c, arma_surface* s, int n, int precision) {
	batch(c, s, n, precision, false);
}
void ma_generate_device(Ctx* c, arma_surface* s, int n, int precision) {
	ma_batch(c, s, n, precision);
}
}  // namespace armab

extern "C" {

int arma_batch_generate(arma_ctx* ctx, arma_surface* surfaces, int n, int precision) {
	return guard([&] {
		ARMA_REQUIRE(ctx && surfaces && n > 0, ARMA_EINVAL, "bad argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		batch(&ctx->c, surfaces, n, precision, false);
	});
}

int arma_batch_generate_host(arma_ctx* ctx, arma_surface* surfaces, int n, int precision) {
	return guard([&] {
		ARMA_REQUIRE(ctx && surfaces && n > 0, ARMA_EINVAL, "bad argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		batch(&ctx->c, surfaces, n, precision, true);
	});
}

namespace {
std::mutex g_tune_mutex;
std::map<std::vector<long long>, arma_tuning> g_tune_cache;

// The batch's shape class: precision, output kind, surface count and the
// sorted multiset of (log2 slice size, length / 32, log2 order size).
std::vector<long long> tune_key(const arma_surface* s, int n, int precision, int host) {
	std::vector<long long> cls;
	for (int k = 0; k < n; ++k) {
		const double area = double(s[k].shape[1]) * s[k].shape[2];
		const double P = double(s[k].order[0]) * s[k].order[1] * s[k].order[2];
		cls.push_back((long long)(std::lround(std::log2(std::max(area, 1.0)))) * 1000000 +
		              (long long)(s[k].shape[0] / 32) * 100 +
		              (long long)std::lround(std::log2(std::max(P, 1.0))));
	}
	std::sort(cls.begin(), cls.end());
	std::vector<long long> key{precision, host, n};
	key.insert(key.end(), cls.begin(), cls.end());
	return key;
}
}  // namespace

int arma_autotune(arma_ctx* ctx, arma_surface* surfaces, int n, int precision, int host,
                  arma_tuning* best_out, double* best_ms) {
	return guard([&] {
		ARMA_REQUIRE(ctx && surfaces && n > 0 && best_out && best_ms, ARMA_EINVAL, "bad argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		const std::vector<long long> key = tune_key(surfaces, n, precision, host);
		{
			std::lock_guard<std::mutex> lk(g_tune_mutex);
			auto it = g_tune_cache.find(key);
			if (it != g_tune_cache.end()) {
				ctx->c.tuning = it->second;
				*best_out = it->second;
				*best_ms = -1.0;
				return;
			}
		}
		auto call = [&] {
			scratch_begin(&ctx->c, 0);
			batch(&ctx->c, surfaces, n, precision, host != 0);
		};
		// wall-clock time per call (every call synchronises before it returns),
		// after one untimed call that builds whatever the setting needs once
		auto time_of = [&](const arma_tuning& t) {
			ctx->c.tuning = t;
			call();
			double best = 1e300;
			for (int r = 0; r < 2; ++r) {
				const auto t0 = std::chrono::steady_clock::now();
				call();
				const auto t1 = std::chrono::steady_clock::now();
				best = std::min(best, std::chrono::duration<double, std::milli>(t1 - t0).count());
			}
			return best;
		};
		arma_tuning cur = ctx->c.tuning;
		double cur_ms = time_of(cur);
		auto consider = [&](arma_tuning t) {
			const double ms = time_of(t);
			if (ms < cur_ms) {
				cur = t;
				cur_ms = ms;
			}
		};
		for (int v : {18, 19, 21})
			if (v != cur.mt_log2_segment) {
				arma_tuning t = cur;
				t.mt_log2_segment = v;
				consider(t);
			}
		if (precision == ARMA_FP32C) {
			for (int a : {1, 2}) {
				arma_tuning t = cur;
				t.ar_ctas_per_sm = a;
				consider(t);
			}
			if (host && n >= 4) {
				const std::pair<int, double> splits[] = {{4, 0.35}, {8, 0.05}, {12, 0.04},
				                                         {12, 0.12}, {16, 0.03}};
				for (const auto& sp : splits) {
					arma_tuning t = cur;
					t.host_groups = sp.first;
					t.host_first = sp.second;
					consider(t);
				}
			}
		}
		ctx->c.tuning = cur;
		*best_out = cur;
		*best_ms = cur_ms;
		std::lock_guard<std::mutex> lk(g_tune_mutex);
		g_tune_cache[key] = cur;
	});
}

namespace {
// The device NIT table of a specification (FP64 values, then FP32), built once
// per context and specification.
const double* nit_table_device(Ctx* c, const arma_nit_table& t, double* x0, double* dx) {
	ARMA_REQUIRE(t.dist == ARMA_NIT_GRAM_CHARLIER || t.dist == ARMA_NIT_SKEW_NORMAL, ARMA_EINVAL,
	             "bad distribution");
	ARMA_REQUIRE(t.stdev > 0.0 && t.lut_nodes >= 4 && t.lut_range > 0.0, ARMA_EINVAL,
	             "bad NIT table");
	const double lo = -t.lut_range * t.stdev;
	*x0 = lo;
	*dx = (t.lut_range * t.stdev - lo) / (t.lut_nodes - 1);
	std::vector<double> key{double(t.dist), t.params[0], t.params[1], t.params[2], t.stdev,
	                        double(t.lut_nodes), t.lut_range};
	auto it = c->nit_tables.find(key);
	if (it != c->nit_tables.end()) return it->second;
	double bx0, bdx;
	std::vector<double> y;
	nit_build_lut(t.dist, t.params, t.stdev, t.lut_nodes, t.lut_range, &bx0, &bdx, y);
	// the FP64 coefficients, then the FP32 ones (4 (nodes + 1) values each)
	const std::vector<double> coef = nit_lut_coefficients(y);
	const std::vector<float> coef_f(coef.begin(), coef.end());
	double* d = nullptr;
	ARMA_CUDA_TRY(cudaMalloc(&d, (sizeof(double) + sizeof(float)) * coef.size()));
	ARMA_CUDA_TRY(cudaMemcpy(d, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice));
	ARMA_CUDA_TRY(cudaMemcpy(d + coef.size(), coef_f.data(), sizeof(float) * coef.size(),
	                         cudaMemcpyHostToDevice));
	c->nit_tables.emplace(key, d);
	return d;
}
}  // namespace

int arma_batch_generate_nit(arma_ctx* ctx, arma_surface* surfaces, int n, int precision,
                            const arma_nit_table* nit) {
	return guard([&] {
		ARMA_REQUIRE(ctx && surfaces && n > 0, ARMA_EINVAL, "bad argument");
		elem_size(precision);
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		std::vector<SurfaceLut> luts(n);
		if (nit)
			for (int k = 0; k < n; ++k) {
				if (nit[k].dist < 0) continue;
				ARMA_REQUIRE(surfaces[k].acf0 > 0.0, ARMA_EINVAL,
				             "NIT needs the variance renormalisation (acf0 > 0)");
				double x0, dx;
				const double* d = nit_table_device(&ctx->c, nit[k], &x0, &dx);
				luts[k].p = precision == ARMA_FP64
				                ? static_cast<const void*>(d)
				                : static_cast<const void*>(d + 4 * size_t(nit[k].lut_nodes + 1));
				luts[k].nodes = nit[k].lut_nodes;
				luts[k].x0 = x0;
				luts[k].inv_dx = 1.0 / dx;
			}
		scratch_begin(&ctx->c, 0);
		batch(&ctx->c, surfaces, n, precision, false, false, luts.data());
	});
}

// ---------------------------------------------------------------- A3'
int arma_ar_fit_choi(const double* acf, int n, int max_order, int determine_order,
                     double var_epsilon, int chop, double* phi_out, int order_out[3],
                     double* var_wn) {
	return guard([&] {
		ARMA_REQUIRE(acf && phi_out && order_out && var_wn, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(n >= 2 && max_order >= 1, ARMA_EINVAL, "bad ACF size or AR order");
		std::vector<double> phi;
		double solver_var = 0.0;
		const int rc = fit_choi(acf, n, max_order, determine_order != 0, var_epsilon, chop != 0,
		                        1e-10, &phi, order_out, &solver_var);
		if (rc == 2) throw Error{ARMA_ENUMERIC, "singular Yule-Walker block"};
		ARMA_REQUIRE(rc == 0, ARMA_EINVAL, "bad ACF size or AR order");
		std::copy(phi.begin(), phi.end(), phi_out);
		const int shape[3] = {n, n, n};
		*var_wn = ar_white_noise_variance(acf, shape, phi.data(), order_out);
	});
}

// ---------------------------------------------------------------- A5
int arma_poly_roots(const double* c, int n, double* re, double* im) {
	return guard([&] {
		ARMA_REQUIRE(c && re && im && n >= 2, ARMA_EINVAL, "null argument or n < 2");
		std::vector<std::complex<double>> roots;
		const int rc = poly_roots(c, n, roots);
		if (rc == 1) throw Error{ARMA_ENUMERIC, "leading term of polynomial must be non-zero"};
		if (rc == 2) throw Error{ARMA_ENUMERIC, "root solving qr method failed to converge"};
		for (int i = 0; i < n - 1; ++i) {
			re[i] = roots[i].real();
			im[i] = roots[i].imag();
		}
	});
}

int arma_validate_process(const double* phi, const int order[3], int* bad_roots) {
	return guard([&] {
		ARMA_REQUIRE(phi && order && bad_roots, ARMA_EINVAL, "null argument");
		require_order(order);
		const int P = order[0] * order[1] * order[2];
		const int rc = validate_ar_process(phi, P, bad_roots);
		if (rc == 1) throw Error{ARMA_ENUMERIC, "leading term of polynomial must be non-zero"};
		if (rc == 2) throw Error{ARMA_ENUMERIC, "root solving qr method failed to converge"};
		if (rc == 3)
			throw Error{ARMA_EINVAL,
			            "AR/MA process is not stationary/invertible: some roots lie inside unit "
			            "circle or on its borderline."};
	});
}

// ---------------------------------------------------------------- M
int arma_ma_fit(const double* acf, const int acf_shape[3], const int order[3],
                double* theta_out, double* var_wn, int* iterations) {
	return guard([&] {
		ARMA_REQUIRE(acf && acf_shape && order && theta_out && var_wn, ARMA_EINVAL,
		             "null argument");
		require_shape(acf_shape, "acf");
		std::vector<double> theta;
		double var = 0.0;
		int it = 0;
		const int rc = ma_fit_fixed_point(acf, acf_shape, order, MaFitOptions{}, &theta, &var, &it,
		                                  nullptr);
		if (rc == 1) throw Error{ARMA_EINVAL, "bad order"};
		if (rc == 2) throw Error{ARMA_ENUMERIC, "bad MA model coefficients"};
		if (rc == 3) throw Error{ARMA_ENUMERIC, "bad white noise variance"};
		std::copy(theta.begin(), theta.end(), theta_out);
		*var_wn = var;
		if (iterations) *iterations = it;
	});
}

int arma_ma_filter(arma_ctx* ctx, const double* theta, const int order[3], const int shape[3],
                   int precision, const void* d_eps, void* d_zeta) {
	return guard([&] {
		ARMA_REQUIRE(ctx && theta && order && shape && d_eps && d_zeta, ARMA_EINVAL,
		             "null argument");
		require_shape(shape, "out_grid");
		require_shape(order, "order");
		const size_t bytes = size_t(shape[0]) * shape[1] * shape[2] * elem_size(precision);
		const char* e = static_cast<const char*>(d_eps);
		const char* z = static_cast<const char*>(d_zeta);
		ARMA_REQUIRE(e + bytes <= z || z + bytes <= e, ARMA_EINVAL, "eps and zeta overlap");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_ma_filter(&ctx->c, theta, order, shape, precision, d_eps, d_zeta);
	});
}

int arma_ma_generate(arma_ctx* ctx, arma_surface* surfaces, int n, int precision) {
	return guard([&] {
		ARMA_REQUIRE(ctx && surfaces && n > 0, ARMA_EINVAL, "bad argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		ma_batch(&ctx->c, surfaces, n, precision);
	});
}

// ---------------------------------------------------------------- driver
struct arma_driver {
	armab::Driver* d;
};

int arma_driver_open(const char* config, int is_path, arma_driver** out) {
	return guard([&] {
		ARMA_REQUIRE(config && out, ARMA_EINVAL, "null argument");
		std::string text;
		if (is_path) {
			std::ifstream f(config);
			if (!f) throw Error{ARMA_EIO, std::string("cannot open ") + config};
			std::ostringstream ss;
			ss << f.rdbuf();
			text = ss.str();
		} else {
			text = config;
		}
		std::unique_ptr<arma_driver> h(new arma_driver{nullptr});
		h->d = driver_open(text);
		*out = h.release();
	});
}

int arma_driver_close(arma_driver* drv) {
	return guard([&] {
		if (!drv) return;
		driver_close(drv->d);
		delete drv;
	});
}

int arma_driver_generate(arma_ctx* ctx, arma_driver* drv) {
	return guard([&] {
		ARMA_REQUIRE(ctx && drv, ARMA_EINVAL, "null argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		driver_generate(&ctx->c, drv->d);
	});
}

int arma_driver_compute_velocity(arma_ctx* ctx, arma_driver* drv) {
	return guard([&] {
		ARMA_REQUIRE(ctx && drv, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(driver_zeta(drv->d), ARMA_EINVAL, "no wavy surface: generate first");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		driver_velocity(&ctx->c, drv->d);
	});
}

int arma_selftest_wait(arma_ctx* ctx) {
	return guard([&] {
		ARMA_REQUIRE(ctx, ARMA_EINVAL, "null argument");
		ARMA_CUDA_TRY(cudaSetDevice(ctx->c.device));
		scratch_begin(&ctx->c, 0);
		launch_wait_selftest(&ctx->c);
		check_device_error(&ctx->c);  // ARMA_ETIMEDOUT, error word cleared
	});
}

int arma_driver_set_output_dir(arma_driver* drv, const char* dir) {
	return guard([&] {
		ARMA_REQUIRE(drv, ARMA_EINVAL, "null argument");
		driver_set_output_dir(drv->d, dir ? dir : "");
	});
}

int arma_driver_write_all(arma_driver* drv, const char* dir) {
	return guard([&] {
		ARMA_REQUIRE(drv, ARMA_EINVAL, "null argument");
		driver_write(drv->d, dir ? dir : "");
	});
}

int arma_driver_info(arma_driver* drv, int shape[3], double delta[3], int order[3],
                     double* var_wn, int vshape[4], unsigned* output_flags) {
	return guard([&] {
		ARMA_REQUIRE(drv, ARMA_EINVAL, "null argument");
		driver_info(drv->d, shape, delta, order, var_wn, vshape, output_flags);
	});
}

int arma_driver_acf(arma_driver* drv, int shape[3], double delta[3], double* out) {
	return guard([&] {
		ARMA_REQUIRE(drv && shape && delta, ARMA_EINVAL, "null argument");
		const double* data = nullptr;
		driver_acf(drv->d, shape, delta, &data);
		if (out && data)
			std::memcpy(out, data, sizeof(double) * size_t(shape[0]) * shape[1] * shape[2]);
	});
}

int arma_driver_copy(arma_driver* drv, int what, double* out) {
	return guard([&] {
		ARMA_REQUIRE(drv && out, ARMA_EINVAL, "null argument");
		int shape[3], order[3], vs[4];
		driver_info(drv->d, shape, nullptr, order, nullptr, vs, nullptr);
		const double* src = nullptr;
		size_t n = 0;
		if (what == 0) {
			src = driver_zeta(drv->d);
			n = size_t(shape[0]) * shape[1] * shape[2];
		} else if (what == 1) {
			src = driver_phi(drv->d);
			n = size_t(order[0]) * order[1] * order[2];
		} else if (what == 2) {
			src = driver_velocity_data(drv->d);
			n = size_t(vs[0]) * vs[1] * vs[2] * vs[3];
		}
		ARMA_REQUIRE(src, ARMA_EINVAL, "nothing to copy (generate / compute first)");
		std::memcpy(out, src, n * sizeof(double));
	});
}

}  // extern "C"
