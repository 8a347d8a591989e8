// Dynamic creation of Mersenne Twister parameter sets (w = 32).
//
// The reference creates the parameter sets of its parallel generators with
// libdcmt's get_mt_parameter_id_st(w, p, id, seed) (src/parallel_mt.hh:199-203,
// driven by src/dcmt.cc:15-33 with p = 521 by default), which follows
// M. Matsumoto and T. Nishimura, "Dynamic Creation of Pseudorandom Number
// Generators" (Monte Carlo and Quasi-Monte Carlo Methods 1998).  libdcmt is not
// part of the reference's tree; this file restates the published method:
//
//   1. Shape.  p is a Mersenne exponent (2^p - 1 prime), nn = ceil(p / 32),
//      rr = 32 nn - p, mm = nn / 2.  The recurrence is
//        x[k+nn] = x[k+mm] ^ ((x[k] & umask) | (x[k+1] & lmask)) A,
//        y A = (y >> 1) ^ (y_0 ? aaa : 0).
//   2. Twist vector.  aaa = 0x80000000 | (r << 16) | id with a 15-bit r; the
//      id makes the characteristic polynomials of different ids different, so
//      generators created with distinct ids are independent.  The top bit is
//      set because the constant term of the characteristic polynomial is that
//      bit.  The 2^15 values of r are visited in an order drawn from `seed`.
//   3. Characteristic polynomial, in closed form (the MT paper, 1998):
//        chi(t) = A^(32-rr) [B^rr + a_0 B^(rr-1) + ... + a_(rr-1)]
//                 + a_rr A^(31-rr) + ... + a_30 A + a_31,
//        A = t^nn + t^mm, B = t^(nn-1) + t^(mm-1),  a_i = bit i of aaa.
//      (Checked against Berlekamp-Massey on the generated sequence for the
//      MT19937 set and random sets of the p = 521 shape.)
//   4. Primitivity.  Since 2^p - 1 is prime, chi is primitive iff it is
//      irreducible, iff t^(2^p) = t mod chi (chi has no root: chi(0) = 1 and
//      chi(1) = 0 is screened).  Most candidates are rejected first by a
//      prescreen: chi mod q for every irreducible q of degree <= 20 is a
//      linear function of the bits of aaa, tabulated once per q.  The
//      survivors take the full test: p squarings mod chi (carry-less
//      Karatsuba products, Barrett reduction).
//   5. Tempering.  y ^= y >> 12; y ^= (y << 7) & b; y ^= (y << 15) & c;
//      y ^= y >> 18.  The masks b, c are chosen bit by bit from the most
//      significant end by a beam search that maximises k(v), the dimension of
//      equidistribution of the top v output bits, at v = 1, 2, ...  k(v) is
//      computed by lattice reduction over F2[z] (Couture, L'Ecuyer and
//      Tezuka; Matsumoto and Nishimura, ACM TOMACS 8(1), 1998): the lattice of
//      the v output-bit series is reduced to a basis with independent leading
//      coefficients, every basis vector carried as a generator state, and
//      k(v) is the smallest basis degree.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include <immintrin.h>
#include <omp.h>

#include "../../include/arma_b200.h"

namespace armab {
namespace dcmt {
namespace {

using Word = uint64_t;

// ----------------------------------------------------------- carry-less products
__attribute__((target("pclmul,sse2"))) inline void clmul_hw(Word a, Word b, Word& lo, Word& hi) {
	const __m128i r = _mm_clmulepi64_si128(_mm_cvtsi64_si128((long long)a),
	                                       _mm_cvtsi64_si128((long long)b), 0x00);
	lo = Word(_mm_cvtsi128_si64(r));
	hi = Word(_mm_cvtsi128_si64(_mm_unpackhi_epi64(r, r)));
}

inline void clmul_sw(Word a, Word b, Word& lo, Word& hi) {
	Word l = 0, h = 0;
	for (int i = 0; i < 64; ++i)
		if ((b >> i) & 1u) {
			l ^= a << i;
			if (i) h ^= a >> (64 - i);
		}
	lo = l;
	hi = h;
}

const bool kHavePclmul = __builtin_cpu_supports("pclmul");

// r[0, na + nb) ^= a * b   (schoolbook)
__attribute__((target("pclmul,sse2"))) void mul_school_hw(const Word* a, size_t na, const Word* b,
                                                         size_t nb, Word* r) {
	for (size_t i = 0; i < na; ++i) {
		if (!a[i]) continue;
		const __m128i ai = _mm_cvtsi64_si128((long long)a[i]);
		for (size_t j = 0; j < nb; ++j) {
			const __m128i p = _mm_clmulepi64_si128(ai, _mm_cvtsi64_si128((long long)b[j]), 0x00);
			r[i + j] ^= Word(_mm_cvtsi128_si64(p));
			r[i + j + 1] ^= Word(_mm_cvtsi128_si64(_mm_unpackhi_epi64(p, p)));
		}
	}
}

void mul_school(const Word* a, size_t na, const Word* b, size_t nb, Word* r) {
	if (kHavePclmul) return mul_school_hw(a, na, b, nb, r);
	for (size_t i = 0; i < na; ++i)
		for (size_t j = 0; j < nb; ++j) {
			Word lo, hi;
			clmul_sw(a[i], b[j], lo, hi);
			r[i + j] ^= lo;
			r[i + j + 1] ^= hi;
		}
}

// r[0, 2n) = a[0, n) * b[0, n); scratch holds at least 8 n words.
void mul_kara(const Word* a, const Word* b, size_t n, Word* r, Word* scratch) {
	if (n <= 24) {
		std::memset(r, 0, sizeof(Word) * 2 * n);
		mul_school(a, n, b, n, r);
		return;
	}
	const size_t h = n / 2, g = n - h;  // low h words, high g >= h words
	Word* sa = scratch;
	Word* sb = sa + g;
	Word* p1 = sb + g;        // 2g
	Word* rest = p1 + 2 * g;  // scratch for the recursion
	// P0 = a0 b0 into r[0, 2h), P2 = a1 b1 into r[2h, 2n)
	mul_kara(a, b, h, r, rest);
	mul_kara(a + h, b + h, g, r + 2 * h, rest);
	for (size_t i = 0; i < g; ++i) {
		sa[i] = a[h + i] ^ (i < h ? a[i] : 0);
		sb[i] = b[h + i] ^ (i < h ? b[i] : 0);
	}
	mul_kara(sa, sb, g, p1, rest);
	// middle = P1 + P0 + P2, added at word offset h
	for (size_t i = 0; i < 2 * h; ++i) p1[i] ^= r[i];
	for (size_t i = 0; i < 2 * g; ++i) p1[i] ^= r[2 * h + i];
	for (size_t i = 0; i < 2 * g; ++i) r[h + i] ^= p1[i];
}

inline int bit_of(const Word* v, long i) { return int((v[i >> 6] >> (i & 63)) & 1u); }
inline void flip(Word* v, long i) { v[i >> 6] ^= Word(1) << (i & 63); }

// dst[0, nw) = src >> sh (bits), reading src[0, nsrc)
void shift_right(const Word* src, size_t nsrc, long sh, Word* dst, size_t nw) {
	const size_t ws = size_t(sh) >> 6;
	const int bs = int(sh & 63);
	for (size_t i = 0; i < nw; ++i) {
		const Word lo = ws + i < nsrc ? src[ws + i] : 0;
		const Word hi = ws + i + 1 < nsrc ? src[ws + i + 1] : 0;
		dst[i] = bs ? (lo >> bs) | (hi << (64 - bs)) : lo;
	}
}

// ------------------------------------------------------ characteristic polynomial
struct Shape {
	int p, nn, mm, rr;
};

Shape shape_of(int p) {
	Shape s;
	s.p = p;
	s.nn = (p + 31) / 32;
	s.rr = 32 * s.nn - p;
	s.mm = s.nn / 2;
	return s;
}

// v *= (t^e1 + t^e2) for a polynomial of `deg` < capacity bits; returns new degree.
long mul_binomial(std::vector<Word>& v, long deg, int e1, int e2) {
	std::vector<Word> out(v.size(), 0);
	auto add_shift = [&](int e) {
		const size_t ws = size_t(e) >> 6;
		const int bs = e & 63;
		const size_t nw = size_t(deg) / 64 + 1;
		for (size_t i = 0; i < nw; ++i) {
			out[ws + i] ^= v[i] << bs;
			if (bs) out[ws + i + 1] ^= v[i] >> (64 - bs);
		}
	};
	add_shift(e1);
	add_shift(e2);
	v.swap(out);
	return deg + std::max(e1, e2);
}

// chi(t) of the set (bit i = coefficient of t^i), p + 1 bits.
std::vector<Word> char_poly(const Shape& s, uint32_t aaa) {
	const size_t nw = size_t(s.p) / 64 + 3;
	std::vector<Word> p1(nw, 0), pa(nw, 0);
	// P1 = Horner in B over (1, a_0, ..., a_(rr-1))
	p1[0] = 1;
	long d1 = 0;
	for (int i = 0; i < s.rr; ++i) {
		d1 = mul_binomial(p1, d1, s.nn - 1, s.mm - 1);
		p1[0] ^= (aaa >> i) & 1u;
	}
	// A^(32 - rr) P1
	for (int i = 0; i < 32 - s.rr; ++i) d1 = mul_binomial(p1, d1, s.nn, s.mm);
	// P2 = Horner in A over (a_rr, ..., a_31)
	long d2 = 0;
	for (int i = s.rr; i < 32; ++i) {
		if (i > s.rr) d2 = mul_binomial(pa, d2, s.nn, s.mm);
		pa[0] ^= (aaa >> i) & 1u;
	}
	for (size_t i = 0; i < nw; ++i) p1[i] ^= pa[i];
	return p1;
}

// ------------------------------------------------------------------- prescreen
constexpr int kScreenDeg = 20;

inline uint32_t mulmod_small(uint32_t a, uint32_t b, uint32_t q, int dq) {
	uint64_t r = 0;
	for (int i = 0; i < dq; ++i)
		if ((b >> i) & 1u) r ^= uint64_t(a) << i;
	for (int i = 2 * dq - 2; i >= dq; --i)
		if ((r >> i) & 1u) r ^= uint64_t(q) << (i - dq);
	return uint32_t(r);
}

uint32_t powt_small(long e, uint32_t q, int dq) {  // t^e mod q
	uint32_t r = 1, b = dq > 1 ? 2u : (2u ^ q);  // t mod q (q = t: 0, q = t + 1: 1)
	while (e) {
		if (e & 1) r = mulmod_small(r, b, q, dq);
		b = mulmod_small(b, b, q, dq);
		e >>= 1;
	}
	return r;
}

struct Screen {
	// per irreducible q: base (constant term contribution incl. the id bits),
	// then E[i] for the 15 free bits of aaa (bits 16..30)
	std::vector<uint32_t> base, free_terms;
	size_t count = 0;
};

// All irreducible polynomials of degree 1..kScreenDeg (bit d = leading term).
const std::vector<uint32_t>& irreducibles() {
	static std::vector<uint32_t> out;
	static std::once_flag once;
	std::call_once(once, [] {
		const uint32_t lim = 1u << (kScreenDeg + 1);
		std::vector<uint8_t> composite(lim, 0);
		for (uint32_t g = 2; g < lim; ++g) {
			if (composite[g]) continue;
			const int dg = 31 - __builtin_clz(g);
			if (dg >= 1) out.push_back(g);
			if (2 * dg > kScreenDeg) continue;
			// mark g * h for deg h >= dg (smaller factors were marked by them)
			for (uint32_t h = 1u << dg; h < (1u << (kScreenDeg - dg + 1)); ++h) {
				uint64_t prod = 0;
				for (int i = 0; i <= kScreenDeg - dg; ++i)
					if ((h >> i) & 1u) prod ^= uint64_t(g) << i;
				if (prod < lim) composite[prod] = 1;
			}
		}
	});
	return out;
}

// The prescreen only rejects candidates that the full test would reject, so
// its degree bound changes the speed, never the result: small p, whose full
// test is cheap, screens with degrees <= 10 only.
Screen make_screen(const Shape& s, uint32_t id_bits) {
	const int max_deg = s.p < 4000 ? 10 : kScreenDeg;
	std::vector<uint32_t> irr;
	for (uint32_t q : irreducibles())
		if (31 - __builtin_clz(q) <= max_deg) irr.push_back(q);
	Screen sc;
	sc.count = irr.size();
	sc.base.resize(irr.size());
	sc.free_terms.resize(irr.size() * 15);
	for (size_t k = 0; k < irr.size(); ++k) {
		const uint32_t q = irr[k];
		const int dq = 31 - __builtin_clz(q);
		const uint32_t A = powt_small(s.nn, q, dq) ^ powt_small(s.mm, q, dq);
		const uint32_t B = powt_small(s.nn - 1, q, dq) ^ powt_small(s.mm - 1, q, dq);
		uint32_t powA[33], powB[33];  // A^j, B^j mod q
		powA[0] = powB[0] = 1;
		for (int j = 1; j <= 32; ++j) {
			powA[j] = mulmod_small(powA[j - 1], A, q, dq);
			powB[j] = mulmod_small(powB[j - 1], B, q, dq);
		}
		const uint32_t Aw = powA[32 - s.rr];
		uint32_t E[32];
		for (int i = 0; i < 32; ++i)
			E[i] = i < s.rr ? mulmod_small(Aw, powB[s.rr - 1 - i], q, dq) : powA[31 - i];
		uint32_t b = mulmod_small(Aw, powB[s.rr], q, dq);
		for (int i = 0; i < 32; ++i)
			if (i < 16 || i == 31) b ^= ((id_bits >> i) & 1u) ? E[i] : 0u;
		sc.base[k] = b;
		for (int i = 0; i < 15; ++i) sc.free_terms[k * 15 + i] = E[16 + i];
	}
	return sc;
}

bool passes_screen(const Screen& sc, uint32_t r15) {
	for (size_t k = 0; k < sc.count; ++k) {
		uint32_t v = sc.base[k];
		const uint32_t* e = &sc.free_terms[k * 15];
		uint32_t bits = r15;
		while (bits) {
			v ^= e[__builtin_ctz(bits)];
			bits &= bits - 1;
		}
		if (v == 0) return false;
	}
	return true;
}

// ------------------------------------------------------------ full primitivity test
// t^(2^p) == t mod chi, by p squarings with Barrett reduction.
bool frobenius_fixes_t(const std::vector<Word>& chi_in, int p) {
	const size_t n = size_t(p) / 64 + 1;  // words holding degree <= p
	std::vector<Word> chi(n + 1, 0);
	std::copy(chi_in.begin(), chi_in.begin() + std::min(chi_in.size(), n + 1), chi.begin());
	// mu = floor(t^(2p) / chi) by long division (degree p)
	std::vector<Word> rem(2 * n + 2, 0), mu(n + 1, 0);
	flip(rem.data(), 2L * p);
	for (long d = 2L * p; d >= p; --d) {
		if (!bit_of(rem.data(), d)) continue;
		const long sh = d - p;
		flip(mu.data(), sh);
		const size_t ws = size_t(sh) >> 6;
		const int bs = int(sh & 63);
		for (size_t i = 0; i <= n; ++i) {
			rem[ws + i] ^= chi[i] << bs;
			if (bs && ws + i + 1 < rem.size()) rem[ws + i + 1] ^= chi[i] >> (64 - bs);
		}
	}
	const size_t m = n + 1;  // operand length for the products
	std::vector<Word> a(m, 0), sq(2 * m, 0), hi(m, 0), qv(2 * m, 0), qq(m, 0), qc(2 * m, 0);
	std::vector<Word> scratch(16 * m + 64);
	std::vector<Word> chim(m, 0), mum(m, 0);
	std::copy(chi.begin(), chi.begin() + std::min(chi.size(), m), chim.begin());
	std::copy(mu.begin(), mu.end(), mum.begin());
	a[0] = 2;  // t
	for (int it = 0; it < p; ++it) {
		// sq = a^2 (degree <= 2p - 2)
		std::fill(sq.begin(), sq.end(), 0);
		for (size_t i = 0; i < n; ++i) {
			Word lo, h2;
			if (kHavePclmul)
				clmul_hw(a[i], a[i], lo, h2);
			else
				clmul_sw(a[i], a[i], lo, h2);
			sq[2 * i] = lo;
			sq[2 * i + 1] = h2;
		}
		// q = ((sq >> p) * mu) >> p
		shift_right(sq.data(), sq.size(), p, hi.data(), m);
		mul_kara(hi.data(), mum.data(), m, qv.data(), scratch.data());
		shift_right(qv.data(), qv.size(), p, qq.data(), m);
		// r = (sq + q chi) mod t^p
		mul_kara(qq.data(), chim.data(), m, qc.data(), scratch.data());
		for (size_t i = 0; i < n; ++i) a[i] = sq[i] ^ qc[i];
		const int top = p & 63;
		a[n - 1] &= top ? (Word(1) << top) - 1 : ~Word(0);
		if (size_t(p) % 64 == 0) a[n - 1] = 0;
		for (size_t i = n; i < m; ++i) a[i] = 0;
	}
	if (a[0] != 2) return false;
	for (size_t i = 1; i < n; ++i)
		if (a[i]) return false;
	return true;
}

// ------------------------------------------------------- equidistribution k(v)
struct Gen {
	const arma_mt_params* p;
	inline uint32_t temper(uint32_t y) const {
		y ^= y >> p->shift0;
		y ^= (y << p->shiftB) & p->maskB;
		y ^= (y << p->shiftC) & p->maskC;
		y ^= y >> p->shift1;
		return y;
	}
};

// A lattice vector: constant part c (v bits; nonzero only for vectors of
// degree 0) plus the output series of a generator state.  For a pure series
// (c == 0) the state is advanced to its first nonzero output, whose index
// is k (degree -(k + 1)) and whose top v bits are lc.
struct LVec {
	uint32_t c = 0;
	std::vector<uint32_t> x;  // ring of nn words
	int i = 0;                // ring index of the oldest word
	long k = 0;
	uint32_t lc = 0;
};

class Lattice {
public:
	Lattice(const arma_mt_params& prm, int v) : prm_(prm), v_(v), gen_{&prm_} {
		top_ = v >= 32 ? 0xffffffffu : ((1u << v) - 1u) << (32 - v);
	}

	// k(v), or -1 when the reduction does not close (a defective generator).
	long run(uint32_t seed) {
		const int n = prm_.nn;
		std::vector<LVec> slot(v_);
		std::vector<bool> used(v_, false);
		for (int j = 0; j < v_; ++j) {
			slot[j].c = 1u << (31 - j);  // e_j: leading coefficient bit 31 - j
			slot[j].x.assign(n, 0);
			slot[j].lc = slot[j].c;
			slot[j].k = -1;  // degree 0
			used[j] = true;
		}
		LVec s0;
		s0.x.assign(n, 0);
		uint32_t st = seed ? seed : 1u;
		for (int j = 0; j < n; ++j) {
			st ^= st << 13;
			st ^= st >> 17;
			st ^= st << 5;
			s0.x[j] = st;
		}
		s0.x[0] &= prm_.umask;
		if (!settle(s0)) return -1;
		LVec cur = std::move(s0);
		for (long guard = 0; guard < 64L * prm_.nn * 32 * (v_ + 2); ++guard) {
			const int piv = __builtin_clz(cur.lc);  // 0 = bit 31
			LVec& u = slot[piv];
			if (deg(u) > deg(cur)) std::swap(u, cur);
			reduce(cur, u);
			if (is_zero(cur)) {
				// k(v) = the smallest -degree of the reduced basis
				long kmin = -1, total = 0;
				for (int j = 0; j < v_; ++j) {
					const long d = -deg(slot[j]);
					total += d;
					kmin = kmin < 0 ? d : std::min(kmin, d);
				}
				const long p = 32L * prm_.nn - prm_.rr;
				if (total != p) return -1;  // the degrees of a basis sum to p
				return kmin;
			}
		}
		return -1;
	}

private:
	static long deg(const LVec& a) { return a.c ? 0 : -(a.k + 1); }

	// the next raw word of the ring, without advancing
	inline uint32_t next_word(const LVec& a) const {
		const int n = prm_.nn;
		const int i1 = a.i + 1 == n ? 0 : a.i + 1;
		int im = a.i + prm_.mm;
		if (im >= n) im -= n;
		const uint32_t y = (a.x[a.i] & prm_.umask) | (a.x[i1] & prm_.lmask);
		return a.x[im] ^ (y >> 1) ^ ((y & 1u) ? prm_.aaa : 0u);
	}
	inline void step(LVec& a) const {
		a.x[a.i] = next_word(a);
		a.i = a.i + 1 == prm_.nn ? 0 : a.i + 1;
	}
	inline uint32_t out(const LVec& a) const { return gen_.temper(next_word(a)) & top_; }

	// a.x ^= b.x with both rings read from their oldest word
	void xor_state(LVec& a, const LVec& b) const {
		const int n = prm_.nn;
		for (int j = 0; j < n; ++j) {
			int ia = a.i + j, ib = b.i + j;
			if (ia >= n) ia -= n;
			if (ib >= n) ib -= n;
			a.x[ia] ^= b.x[ib];
		}
	}

	// Advance a pure series to its first nonzero output; false if it is zero.
	bool settle(LVec& a) const {
		if (a.c) {
			a.lc = a.c;
			return true;
		}
		long steps = 0;
		for (;;) {
			const uint32_t o = out(a);
			if (o) {
				a.lc = o;
				return true;
			}
			step(a);
			++a.k;
			if (++steps % (4 * prm_.nn) == 0) {
				bool zero = true;
				for (int j = 0; j < prm_.nn && zero; ++j)
					zero = (j == 0 ? (a.x[a.i] & prm_.umask) : a.x[(a.i + j) % prm_.nn]) == 0;
				if (zero) {
					a.lc = 0;
					return false;
				}
			}
		}
	}

	bool is_zero(const LVec& a) const { return a.c == 0 && a.lc == 0; }

	// a += z^(deg a - deg b) b, deg a >= deg b, same leading pivot
	void reduce(LVec& a, const LVec& b) const {
		if (a.c && b.c) {  // both degree 0
			a.c ^= b.c;
			xor_state(a, b);
			if (a.c) {
				a.lc = a.c;
				return;
			}
			a.k = 0;
			settle(a);
			return;
		}
		if (a.c) {  // a degree 0, b pure series: z^(k_b + 1) b = lc_b + series of B * state_b
			LVec tb = b;
			step(tb);
			a.c ^= b.lc;
			xor_state(a, tb);
			if (a.c) {
				a.lc = a.c;
				return;
			}
			a.k = 0;
			settle(a);
			return;
		}
		// both pure series, advanced to their leading outputs: states align
		xor_state(a, b);
		const uint32_t o = a.lc ^ b.lc;
		if (o) {
			a.lc = o;
			return;
		}
		step(a);
		++a.k;
		settle(a);
	}

	arma_mt_params prm_;
	int v_;
	Gen gen_;
	uint32_t top_;
};

}  // namespace

// The shape (nn, mm, rr) of a parameter set of period 2^p - 1.
bool mersenne_exponent(int p) {
	static const int kExp[] = {521, 607, 1279, 2203, 2281, 3217, 4253, 4423, 9689, 9941, 11213,
	                           19937, 21701, 23209, 44497};
	for (int e : kExp)
		if (e == p) return true;
	return false;
}

bool is_primitive(const arma_mt_params& prm) {
	const Shape s{32 * prm.nn - prm.rr, prm.nn, prm.mm, prm.rr};
	if (!((prm.aaa >> 31) & 1u)) return false;
	const std::vector<Word> chi = char_poly(s, prm.aaa);
	if (!bit_of(chi.data(), 0)) return false;
	int ones = 0;  // chi(1)
	for (Word w : chi) ones ^= __builtin_parityll(w);
	if (!ones) return false;
	return frobenius_fixes_t(chi, s.p);
}

long equidistribution(const arma_mt_params& prm, int v) {
	Lattice lat(prm, v);
	return lat.run(0x9e3779b9u ^ uint32_t(v));
}

namespace {

void base_params(const Shape& s, arma_mt_params* o) {
	std::memset(o, 0, sizeof(*o));
	o->mm = s.mm;
	o->nn = s.nn;
	o->rr = s.rr;
	o->ww = 32;
	o->wmask = 0xffffffffu;
	o->umask = s.rr == 32 ? 0u : (0xffffffffu << s.rr);
	o->lmask = ~o->umask;
	o->shift0 = 12;
	o->shiftB = 7;
	o->shiftC = 15;
	o->shift1 = 18;
	o->i = s.nn;
}

// Tempering search, a beam search over the mask bits from the most
// significant output bit down.  Output bit j (bits 31..32-v are the top v)
// is, for j >= 32 - l, bit j of y3 = y2 ^ ((y2 << t) & c), which involves c_j
// and bit j - t of y2 = y1 ^ ((y1 << s) & b), i.e. b_j and b_(j-t).  At step v
// (j = 32 - v) the bits among b_j, c_j and b_(j-t) that earlier steps have
// not set are set in every way for each of the kBeam best partial masks of
// step v - 1, k(v) is computed for each, and the kBeam best by
// (k(v), k(1) + ... + k(v-1)) are kept; bits that act on no output bit above
// j stay free for later steps.  Ties keep the earlier candidate, so the
// result depends only on the twist vector.
constexpr int kBeam = 64;

struct Partial {
	uint32_t b = 0, c = 0;
	long kv = 0, ksum = 0;
};

void search_tempering(arma_mt_params* prm) {
	const int sb = prm->shiftB, tc = prm->shiftC, l = prm->shift1;
	std::vector<Partial> beam(1);
	uint32_t done_b = 0, done_c = 0;  // mask bits already decided
	for (int v = 1; v <= 32; ++v) {
		const int j = 32 - v;
		if (j < 32 - l) break;  // below: y ^= y >> l mixes in higher bits
		uint32_t nb = 0, nc = 0;  // bits decided at this step
		if (j >= sb) nb |= 1u << j;
		if (j >= tc) nc |= 1u << j;
		if (j - tc >= sb) nb |= 1u << (j - tc);
		nb &= ~done_b;
		nc &= ~done_c;
		std::vector<int> bits;  // 0..31: b bit, 32..63: c bit
		for (int i = 0; i < 32; ++i) {
			if ((nb >> i) & 1u) bits.push_back(i);
			if ((nc >> i) & 1u) bits.push_back(32 + i);
		}
		if (bits.empty()) continue;
		std::vector<Partial> cand;
		for (const Partial& q : beam)
			for (uint32_t combo = 0; combo < (1u << bits.size()); ++combo) {
				Partial n = q;
				n.ksum = q.ksum + q.kv;
				for (size_t k = 0; k < bits.size(); ++k)
					if ((combo >> k) & 1u) {
						if (bits[k] < 32)
							n.b |= 1u << bits[k];
						else
							n.c |= 1u << (bits[k] - 32);
					}
				cand.push_back(n);
			}
#pragma omp parallel for schedule(dynamic, 1)
		for (long i = 0; i < long(cand.size()); ++i) {
			arma_mt_params t = *prm;
			t.maskB = cand[size_t(i)].b;
			t.maskC = cand[size_t(i)].c;
			cand[size_t(i)].kv = equidistribution(t, v);
		}
		std::stable_sort(cand.begin(), cand.end(), [](const Partial& x, const Partial& y) {
			return x.kv != y.kv ? x.kv > y.kv : x.ksum > y.ksum;
		});
		if (cand.size() > size_t(kBeam)) cand.resize(kBeam);
		beam.swap(cand);
		done_b |= nb;
		done_c |= nc;
	}
	prm->maskB = beam.front().b;
	prm->maskC = beam.front().c;
}

}  // namespace

int create(int p, int id, uint32_t seed, arma_mt_params* out) {
	const Shape s = shape_of(p);
	uint32_t id_bits = 0x80000000u | uint32_t(id);
	const Screen sc = make_screen(s, id_bits);
	// visit the 2^15 values of the free bits in a seeded order
	std::vector<uint32_t> order(1u << 15);
	std::iota(order.begin(), order.end(), 0u);
	std::mt19937 rng(seed);
	std::shuffle(order.begin(), order.end(), rng);
	std::vector<uint32_t> survivors;
	for (uint32_t r : order)
		if (passes_screen(sc, r)) survivors.push_back(r);
	const int nth = std::max(1, omp_get_max_threads());
	for (size_t base = 0; base < survivors.size(); base += size_t(nth)) {
		const size_t cnt = std::min(size_t(nth), survivors.size() - base);
		std::vector<uint8_t> ok(cnt, 0);
#pragma omp parallel for schedule(dynamic, 1)
		for (long j = 0; j < long(cnt); ++j) {
			const uint32_t aaa = id_bits | (survivors[base + size_t(j)] << 16);
			ok[size_t(j)] = frobenius_fixes_t(char_poly(s, aaa), s.p) ? 1 : 0;
		}
		for (size_t j = 0; j < cnt; ++j) {
			if (!ok[j]) continue;
			base_params(s, out);
			out->aaa = id_bits | (survivors[base + j] << 16);
			search_tempering(out);
			return 0;
		}
	}
	return -1;
}

}  // namespace dcmt
}  // namespace armab
