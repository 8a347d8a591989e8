// Replica router: one serving replica (arma_server) per listed device behind
// one handle.  Streams are independent, so the surface streams of a node
// shard across GPUs with no exchange at all; the router only places each
// stream, forwards its requests and merges the replicas' completions.
//
// Placement: the replica with the least stream state placed on it, measured
// as nx * ny * (pt - 1 + 2 T) points (the two slice buffers of a stream's
// device state, which dominate its HBM footprint), ties to the replica with
// fewer streams, then to the lower index.  A stream stays on its replica for
// life (its history slices and MT window live there).
//
// Ids: the replica's own stream and request ids with the replica index in the
// top 8 bits.  Polling drains every replica without waiting, starting at a
// rotating replica so that none is starved; when nothing is ready it waits on
// one replica at a time in steps of at most a millisecond until the deadline.
#include <algorithm>
#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "internal.h"

struct arma_router {
	struct Replica {
		int device = 0;
		arma_server* srv = nullptr;
		unsigned long long placed = 0;  // points of stream state placed here
		int streams = 0;
	};
	std::vector<Replica> reps;
	std::map<uint64_t, unsigned long long> weight;  // open stream -> its placed points
	int chunk_slices = 0;
	int next_poll = 0;
	std::mutex mu;
};

namespace {

constexpr int kReplicaShift = 56;
constexpr int kMaxReplicas = 256;

uint64_t global_id(int replica, uint64_t local) {
	return (uint64_t(replica) << kReplicaShift) | local;
}

int replica_of(const arma_router* r, uint64_t id) {
	const int k = int(id >> kReplicaShift);
	ARMA_REQUIRE(k < int(r->reps.size()), ARMA_EINVAL, "unknown stream");
	return k;
}

uint64_t local_of(uint64_t id) { return id & ((uint64_t(1) << kReplicaShift) - 1); }

// rc of a replica call: its error as this call's error (the message is already
// the thread's last error)
void forward(int rc) {
	if (rc != ARMA_OK) throw armab::Error{rc, armab::last_error()};
}

}  // namespace

extern "C" {

int arma_router_create(const int* devices, int n, const arma_server_config* cfg,
                       arma_router** out) {
	return armab::guard([&] {
		ARMA_REQUIRE(devices && cfg && out, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(n >= 1 && n <= kMaxReplicas, ARMA_EINVAL, "replicas must be in [1, 256]");
		std::unique_ptr<arma_router> r(new arma_router());
		r->chunk_slices = cfg->chunk_slices;
		r->reps.resize(n);
		try {
			for (int k = 0; k < n; ++k) {
				r->reps[k].device = devices[k];
				forward(arma_server_create(devices[k], cfg, &r->reps[k].srv));
			}
		} catch (...) {
			for (auto& rep : r->reps)
				if (rep.srv) arma_server_destroy(rep.srv);
			throw;
		}
		*out = r.release();
	});
}

int arma_router_destroy(arma_router* r) {
	return armab::guard([&] {
		if (!r) return;
		int rc = ARMA_OK;
		for (auto& rep : r->reps)
			if (rep.srv) {
				const int k = arma_server_destroy(rep.srv);
				if (rc == ARMA_OK) rc = k;
			}
		delete r;
		forward(rc);
	});
}

int arma_router_replicas(arma_router* r, int* n) {
	return armab::guard([&] {
		ARMA_REQUIRE(r && n, ARMA_EINVAL, "null argument");
		*n = int(r->reps.size());
	});
}

int arma_router_stream_open(arma_router* r, const arma_stream_spec* spec, uint64_t* stream_id) {
	return armab::guard([&] {
		ARMA_REQUIRE(r && spec && stream_id, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(spec->nx > 0 && spec->ny > 0 && spec->order[0] > 0, ARMA_EINVAL,
		             "Bad \"stream\": dimensions must be positive");
		const unsigned long long w = (unsigned long long)spec->nx * spec->ny *
		                             (unsigned long long)(spec->order[0] - 1 + 2 * r->chunk_slices);
		std::lock_guard<std::mutex> lk(r->mu);
		int best = 0;
		for (int k = 1; k < int(r->reps.size()); ++k) {
			const auto& a = r->reps[k];
			const auto& b = r->reps[best];
			if (a.placed < b.placed || (a.placed == b.placed && a.streams < b.streams)) best = k;
		}
		uint64_t local = 0;
		forward(arma_stream_open(r->reps[best].srv, spec, &local));
		ARMA_REQUIRE(local >> kReplicaShift == 0, ARMA_EINVAL, "replica stream id out of range");
		const uint64_t id = global_id(best, local);
		r->reps[best].placed += w;
		r->reps[best].streams += 1;
		r->weight[id] = w;
		*stream_id = id;
	});
}

int arma_router_stream_close(arma_router* r, uint64_t stream_id) {
	return armab::guard([&] {
		ARMA_REQUIRE(r, ARMA_EINVAL, "null argument");
		std::lock_guard<std::mutex> lk(r->mu);
		auto it = r->weight.find(stream_id);
		ARMA_REQUIRE(it != r->weight.end(), ARMA_EINVAL, "unknown stream");
		const int k = replica_of(r, stream_id);
		forward(arma_stream_close(r->reps[k].srv, local_of(stream_id)));
		r->reps[k].placed -= it->second;
		r->reps[k].streams -= 1;
		r->weight.erase(it);
	});
}

int arma_router_stream_submit(arma_router* r, uint64_t stream_id, float* zeta_out,
                              float* velocity_out, uint64_t* request_id) {
	return armab::guard([&] {
		ARMA_REQUIRE(r, ARMA_EINVAL, "null argument");
		int k;
		{
			std::lock_guard<std::mutex> lk(r->mu);
			ARMA_REQUIRE(r->weight.count(stream_id), ARMA_EINVAL, "unknown stream");
			k = replica_of(r, stream_id);
		}
		uint64_t local = 0;
		forward(arma_stream_submit(r->reps[k].srv, local_of(stream_id), zeta_out, velocity_out,
		                           &local));
		if (request_id) *request_id = global_id(k, local);
	});
}

int arma_router_poll(arma_router* r, arma_completion* out, int max, int timeout_ms, int* n) {
	return armab::guard([&] {
		ARMA_REQUIRE(r && out && n && max > 0, ARMA_EINVAL, "null argument");
		using Clock = std::chrono::steady_clock;
		const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(timeout_ms, 0));
		const int R = int(r->reps.size());
		int start;
		{
			std::lock_guard<std::mutex> lk(r->mu);
			start = r->next_poll;
			r->next_poll = (r->next_poll + 1) % R;
		}
		auto drain = [&](int first, int wait_ms) {
			int k = 0;
			for (int q = 0; q < R && k < max; ++q) {
				const int rep = (first + q) % R;
				int m = 0;
				forward(arma_server_poll(r->reps[rep].srv, out + k, max - k, q == 0 ? wait_ms : 0, &m));
				for (int j = k; j < k + m; ++j) {
					out[j].request = global_id(rep, out[j].request);
					out[j].stream = global_id(rep, out[j].stream);
				}
				k += m;
			}
			return k;
		};
		int k = drain(start, 0);
		for (int turn = 1; k == 0 && timeout_ms != 0; ++turn) {
			int step = 1;
			if (timeout_ms > 0) {
				const auto left = std::chrono::duration_cast<std::chrono::milliseconds>(
				    deadline - Clock::now()).count();
				if (left <= 0) break;
				step = int(std::min<long long>(left, 1));
			}
			k = drain((start + turn) % R, step);
		}
		*n = k;
	});
}

int arma_router_placement(arma_router* r, uint64_t stream_id, int* replica, int* device) {
	return armab::guard([&] {
		ARMA_REQUIRE(r && replica && device, ARMA_EINVAL, "null argument");
		std::lock_guard<std::mutex> lk(r->mu);
		ARMA_REQUIRE(r->weight.count(stream_id), ARMA_EINVAL, "unknown stream");
		*replica = replica_of(r, stream_id);
		*device = r->reps[*replica].device;
	});
}

int arma_router_stats_get(arma_router* r, int replica, arma_server_stats* out) {
	return armab::guard([&] {
		ARMA_REQUIRE(r && out, ARMA_EINVAL, "null argument");
		ARMA_REQUIRE(replica >= 0 && replica < int(r->reps.size()), ARMA_EINVAL,
		             "replica out of range");
		forward(arma_server_stats_get(r->reps[replica].srv, out));
	});
}

}  // extern "C"
