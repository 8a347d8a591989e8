// Oracle (test infrastructure): dcmt Mersenne Twister restatement, mt.dat
// file IO and the libstdc++ normal white noise.
#include "oracle.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <random>
#include <vector>

namespace {

// On-disk record of one dcmt parameter set: the raw x86-64 mt_struct
// (fifteen 32-bit fields, 4 bytes of padding and the state pointer) as the
// reference writes it with `out.write((char*)&rhs, sizeof(mt_config))`
// (src/parallel_mt.hh:99-104), followed by nn 32-bit state words.
constexpr size_t kRecordHeader = 72;

// The dcmt generator state: parameters plus the nn-word state array.
struct Mt {
	orc_mt_params p;
	std::vector<uint32_t> st;
	int i = 0;

	// sgenrand_mt: Knuth's multiplier 1812433253 initialisation, masked by
	// wmask (dcmt; called by parallel_mt::init, src/parallel_mt.hh:258-260).
	void seed(uint32_t s) {
		st.assign(p.nn, 0);
		for (int k = 0; k < p.nn; ++k) {
			st[k] = s;
			s = 1812433253u * (s ^ (s >> 30)) + uint32_t(k + 1);
		}
		i = p.nn;
		for (int k = 0; k < p.nn; ++k) st[k] &= p.wmask;
	}

	// genrand_mt: the MT linear recurrence over the whole array, then
	// tempering (dcmt; called by parallel_mt::operator(),
	// src/parallel_mt.hh:236).
	uint32_t next() {
		const int n = p.nn, m = p.mm;
		if (i >= n) {
			const uint32_t u = p.umask, l = p.lmask, a = p.aaa;
			int k = 0;
			for (; k < n - m; ++k) {
				const uint32_t x = (st[k] & u) | (st[k + 1] & l);
				st[k] = st[k + m] ^ (x >> 1) ^ ((x & 1u) ? a : 0u);
			}
			for (; k < n - 1; ++k) {
				const uint32_t x = (st[k] & u) | (st[k + 1] & l);
				st[k] = st[k + m - n] ^ (x >> 1) ^ ((x & 1u) ? a : 0u);
			}
			const uint32_t x = (st[n - 1] & u) | (st[0] & l);
			st[n - 1] = st[m - 1] ^ (x >> 1) ^ ((x & 1u) ? a : 0u);
			i = 0;
		}
		uint32_t y = st[i++];
		y ^= y >> p.shift0;
		y ^= (y << p.shiftB) & p.maskB;
		y ^= (y << p.shiftC) & p.maskC;
		y ^= y >> p.shift1;
		return y;
	}
};

// UniformRandomBitGenerator adaptor with the same result_type/min/max as the
// reference's parallel_mt (src/parallel_mt.hh:217-275), so that libstdc++'s
// generate_canonical consumes exactly two words per uniform.
struct Urbg {
	using result_type = uint32_t;
	Mt* mt;
	size_t used = 0;
	static constexpr result_type min() { return 0; }
	static constexpr result_type max() { return std::numeric_limits<uint32_t>::max(); }
	result_type operator()() { ++used; return mt->next(); }
};

}  // namespace

extern "C" void orc_mt19937_params(orc_mt_params* p) {
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
}

extern "C" void orc_mt_sgenrand(const orc_mt_params* p, uint32_t seed,
                                uint32_t* state) {
	Mt mt;
	mt.p = *p;
	mt.seed(seed);
	std::memcpy(state, mt.st.data(), sizeof(uint32_t) * p->nn);
}

extern "C" void orc_mt_genrand(const orc_mt_params* p, uint32_t seed, size_t n,
                               uint32_t* out) {
	Mt mt;
	mt.p = *p;
	mt.seed(seed);
	for (size_t k = 0; k < n; ++k) out[k] = mt.next();
}

extern "C" void orc_std_mt19937(uint32_t seed, size_t n, uint32_t* out) {
	std::mt19937 g(seed);
	for (size_t k = 0; k < n; ++k) out[k] = uint32_t(g());
}

// Reference: src/parallel_mt.hh:90-97 (operator>>) and
// src/parallel_mt.cc:28-59 (read_parallel_mts counts records until EOF).
extern "C" int orc_mt_file_count(const char* path) {
	std::ifstream in(path, std::ios::binary);
	if (!in) return -1;
	int n = 0;
	for (;;) {
		unsigned char hdr[kRecordHeader];
		if (!in.read(reinterpret_cast<char*>(hdr), kRecordHeader)) break;
		int32_t nn;
		std::memcpy(&nn, hdr + 8, 4);
		if (nn <= 0 || nn > (1 << 20)) return -2;
		in.seekg(std::streamoff(nn) * 4, std::ios::cur);
		if (!in) break;
		++n;
	}
	return n;
}

extern "C" int orc_mt_file_read(const char* path, int index, orc_mt_params* p) {
	std::ifstream in(path, std::ios::binary);
	if (!in) return -1;
	for (int k = 0;; ++k) {
		unsigned char hdr[kRecordHeader];
		if (!in.read(reinterpret_cast<char*>(hdr), kRecordHeader)) return -3;
		std::memcpy(p, hdr, sizeof(orc_mt_params));  // 60 bytes of fields
		if (p->nn <= 0 || p->nn > (1 << 20)) return -2;
		in.seekg(std::streamoff(p->nn) * 4, std::ios::cur);
		if (!in) return -3;
		if (k == index) return 0;
	}
}

extern "C" int orc_mt_file_write(const char* path, const orc_mt_params* p, int n,
                                 const uint32_t* states) {
	std::ofstream out(path, std::ios::binary);
	if (!out) return -1;
	size_t off = 0;
	for (int k = 0; k < n; ++k) {
		unsigned char hdr[kRecordHeader] = {0};
		std::memcpy(hdr, &p[k], sizeof(orc_mt_params));
		out.write(reinterpret_cast<const char*>(hdr), kRecordHeader);
		out.write(reinterpret_cast<const char*>(states + off), std::streamsize(p[k].nn) * 4);
		off += size_t(p[k].nn);
	}
	return out ? 0 : -4;
}

// Reference: src/white_noise.hh:23-58 (sequential build: every value is
// drawn from mts[0] in C order) with the distribution constructed at
// src/generator/basic_arma_model.cc:43-47.  libstdc++'s normal_distribution
// (Marsaglia polar method over generate_canonical) is used as-is.
extern "C" void orc_white_noise(const orc_mt_params* p, uint32_t seed,
                                double stddev, size_t n, double* out) {
	Mt mt;
	mt.p = *p;
	mt.seed(seed);
	Urbg g{&mt};
	std::normal_distribution<double> dist(0.0, stddev);
	for (size_t k = 0; k < n; ++k) out[k] = dist(g);
}

extern "C" size_t orc_white_noise_words(const orc_mt_params* p, uint32_t seed,
                                        size_t n) {
	Mt mt;
	mt.p = *p;
	mt.seed(seed);
	Urbg g{&mt};
	std::normal_distribution<double> dist(0.0, 1.0);
	for (size_t k = 0; k < n; ++k) (void)dist(g);
	return g.used;
}
