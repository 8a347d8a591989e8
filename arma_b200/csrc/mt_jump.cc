// Host-side GF(2) polynomial arithmetic for jumping a dcmt Mersenne Twister
// stream ahead.
//
// The essential state of a w=32 dcmt generator has p = 32*nn - rr bits and
// evolves by an invertible linear map A over GF(2).  Every bit of the raw
// word sequence x[j] (sgenrand_mt's state followed by the recurrence) is a
// fixed linear functional of the state, so all of them satisfy the
// characteristic polynomial phi(t) of A.  For a jump of J words:
//     g(t) = t^J mod phi(t)   =>   x[J + w] = XOR_{i : g_i = 1} x[i + w]
// for w >= 1 (and the upper 32-rr bits of w = 0), i.e. the window of nn words
// J positions ahead is an XOR of windows of the raw sequence.  phi is found by
// Berlekamp-Massey on 2p bits of one bit position of the raw sequence (its
// minimal polynomial has degree p when phi is primitive, as it is for
// MT19937 and for dcmt-created sets); t^J for J = 2^q comes from q modular
// squarings.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "internal.h"

namespace armab {
namespace {

using Bits = std::vector<uint64_t>;

inline int get_bit(const Bits& b, long i) { return int((b[size_t(i) >> 6] >> (i & 63)) & 1u); }
inline void flip_bit(Bits& b, long i) { b[size_t(i) >> 6] ^= uint64_t(1) << (i & 63); }

// 64 bits of b starting at bit `off` (bits beyond the end read as 0).
inline uint64_t word_at(const Bits& b, long off) {
	const size_t w = size_t(off) >> 6;
	const int s = int(off & 63);
	const uint64_t lo = w < b.size() ? b[w] : 0;
	if (s == 0) return lo;
	const uint64_t hi = (w + 1) < b.size() ? b[w + 1] : 0;
	return (lo >> s) | (hi << (64 - s));
}

// a ^= b << sh  (a sized to hold the result)
void xor_shifted(Bits& a, const Bits& b, long sh, long nbits_b) {
	const size_t ws = size_t(sh) >> 6;
	const int bs = int(sh & 63);
	const size_t nw = (size_t(nbits_b) + 63) >> 6;
	for (size_t i = 0; i < nw; ++i) {
		const uint64_t v = i < b.size() ? b[i] : 0;
		if (ws + i < a.size()) a[ws + i] ^= v << bs;
		if (bs && ws + i + 1 < a.size()) a[ws + i + 1] ^= v >> (64 - bs);
	}
}

// Raw words x[0..count) of the dcmt recurrence from the seeded state.
std::vector<uint32_t> raw_words(const arma_mt_params& p, uint32_t seed, size_t count) {
	const int n = p.nn, m = p.mm;
	std::vector<uint32_t> x(count);
	uint32_t s = seed;
	for (int k = 0; k < n && size_t(k) < count; ++k) {
		x[k] = s & p.wmask;
		s = 1812433253u * (s ^ (s >> 30)) + uint32_t(k + 1);
	}
	for (size_t j = n; j < count; ++j) {
		const uint32_t y = (x[j - n] & p.umask) | (x[j - n + 1] & p.lmask);
		x[j] = x[j - n + m] ^ (y >> 1) ^ ((y & 1u) ? p.aaa : 0u);
	}
	return x;
}

// Berlekamp-Massey over GF(2).  Returns the characteristic polynomial (bit i
// = coefficient of t^i) and its degree.
Bits berlekamp_massey(const std::vector<uint8_t>& s, int* degree) {
	const long N = long(s.size());
	const size_t nw = size_t(N + 64) / 64 + 1;
	Bits C(nw, 0), B(nw, 0), T;
	C[0] = B[0] = 1;
	// reversed sequence: r bit j = s[N-1-j], so s[n-i] = r[(N-1-n) + i]
	Bits r(nw, 0);
	for (long j = 0; j < N; ++j)
		if (s[N - 1 - j]) flip_bit(r, j);
	long L = 0, m = 1;
	for (long n = 0; n < N; ++n) {
		// d = s[n] + sum_{i=1..L} C_i s[n-i] = parity(C & r>>(N-1-n)) over bits 0..L
		uint64_t acc = 0;
		const long base = N - 1 - n;
		const size_t words = size_t(L + 64) / 64;
		for (size_t w = 0; w < words; ++w) {
			uint64_t c = C[w];
			if (w == words - 1) {
				const int rem = int((L + 1) - long(w) * 64);
				if (rem < 64) c &= (uint64_t(1) << rem) - 1;
			}
			acc ^= c & word_at(r, base + long(w) * 64);
		}
		const int d = __builtin_parityll(acc);
		if (d == 0) {
			++m;
		} else if (2 * L <= n) {
			T = C;
			xor_shifted(C, B, m, long(B.size()) * 64);
			L = n + 1 - L;
			B = T;
			m = 1;
		} else {
			xor_shifted(C, B, m, long(B.size()) * 64);
			++m;
		}
	}
	// phi(t) = t^L C(1/t): coefficient of t^(L-i) is C_i
	Bits phi(size_t(L) / 64 + 1, 0);
	for (long i = 0; i <= L; ++i)
		if (get_bit(C, i)) flip_bit(phi, L - i);
	*degree = int(L);
	return phi;
}

// Reduction context: phi and its 64 bit-shifted copies.
struct Reducer {
	int p;
	std::vector<Bits> shifted;  // shifted[s] = phi << s, sized for aligned XOR
	explicit Reducer(const Bits& phi, int deg) : p(deg), shifted(64) {
		const size_t nw = size_t(deg) / 64 + 2;
		for (int s = 0; s < 64; ++s) {
			shifted[s].assign(nw, 0);
			xor_shifted(shifted[s], phi, s, deg + 1);
		}
	}
	// a (degree < 2p) mod phi, in place; result has degree < p
	void reduce(Bits& a) const {
		for (long d = 2L * p - 2; d >= p; --d) {
			if (!get_bit(a, d)) continue;
			const long sh = d - p;
			const Bits& ph = shifted[sh & 63];
			const size_t ws = size_t(sh) >> 6;
			for (size_t i = 0; i < ph.size() && ws + i < a.size(); ++i) a[ws + i] ^= ph[i];
		}
	}
	Bits square(const Bits& a) const {
		Bits r(size_t(2 * p) / 64 + 2, 0);
		for (long i = 0; i < p; ++i)
			if (get_bit(a, i)) flip_bit(r, 2 * i);
		reduce(r);
		r.resize(size_t(p) / 64 + 1);
		return r;
	}
};

}  // namespace

bool mt_jump_tables(const arma_mt_params& prm, int log2_jump, int levels,
                    std::vector<std::vector<int32_t>>* set_bits, int* degree) {
	const int p = 32 * prm.nn - prm.rr;
	// 2p bits of bit 0 of the raw sequence, starting past the seeded words
	const size_t start = size_t(prm.nn);
	std::vector<uint32_t> x = raw_words(prm, 4357u, start + 2 * size_t(p) + 8);
	std::vector<uint8_t> s(2 * size_t(p));
	for (size_t j = 0; j < s.size(); ++j) s[j] = uint8_t(x[start + j] & 1u);
	int L = 0;
	Bits phi = berlekamp_massey(s, &L);
	*degree = L;
	if (L != p) return false;  // not a full-period set: the caller generates sequentially
	Reducer red(phi, p);
	Bits g(size_t(p) / 64 + 1, 0);
	flip_bit(g, 1);  // t
	for (int q = 0; q < log2_jump; ++q) g = red.square(g);
	set_bits->assign(levels, {});
	for (int lv = 0; lv < levels; ++lv) {
		auto& v = (*set_bits)[lv];
		for (long i = 0; i < p; ++i)
			if (get_bit(g, i)) v.push_back(int32_t(i));
		g = red.square(g);
	}
	return true;
}

}  // namespace armab
