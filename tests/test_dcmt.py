"""dcmt parameter-set creation (``arma_mt_create``) and the committed sets.

The reference creates its generators' parameter sets with libdcmt
(get_mt_parameter_id_st, src/parallel_mt.hh:199-203; arma-dcmt,
src/dcmt.cc:15-33), which is not part of its tree.  These tests pin the
library's creator and the committed files without it:

  * known answers: MT19937 is primitive, and its dimensions of
    equidistribution k(v) are the published ones (k(v) = 623 for v >= 17,
    total defect sum_v (floor(19937 / v) - k(v)) = 6750);
  * primitivity of every committed p = 521 set is re-checked here in pure
    Python, independently of the library: Berlekamp-Massey on the raw
    sequence gives the characteristic polynomial, then t^(2^p) = t mod it;
    the same check agrees with the library's verdict on random twist vectors;
  * k(v) of a committed set equals the rank computation over GF(2) of the
    output bits as linear functions of the state;
  * the creator is deterministic in (p, id, seed) and reproduces the
    committed files' sets.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import arma_b200 as A
from arma_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "arma_b200", "data")
MT19937_FILE = os.path.join(DATA, "mt.dat")
MT521_FILE = os.path.join(DATA, "mt521.dat")


def read_sets(path):
    return [A.mt_file_read(path, k) for k in range(A.mt_file_count(path))]


# ----------------------------------------------------------- pure-Python GF(2)
def raw_words(p, seed, count):
    """The raw (untempered) word sequence of the set: sgenrand_mt's state,
    then the recurrence."""
    nn, mm = p.nn, p.mm
    x, s = [], seed
    for k in range(nn):
        x.append(s & p.wmask)
        s = (1812433253 * (s ^ (s >> 30)) + k + 1) & 0xFFFFFFFF
    for j in range(nn, count):
        y = (x[j - nn] & p.umask) | (x[j - nn + 1] & p.lmask)
        x.append(x[j - nn + mm] ^ (y >> 1) ^ (p.aaa if y & 1 else 0))
    return x


def berlekamp_massey(bits):
    """Characteristic polynomial (int, bit i = coefficient of t^i) and its
    degree for a GF(2) sequence."""
    c, b, L, m = 1, 1, 0, 1
    for n in range(len(bits)):
        d = bits[n]
        cc, i = c >> 1, 1
        while cc:
            if cc & 1:
                d ^= bits[n - i]
            cc >>= 1
            i += 1
        if d == 0:
            m += 1
        elif 2 * L <= n:
            c, b, L, m = c ^ (b << m), c, n + 1 - L, 1
        else:
            c ^= b << m
            m += 1
    phi = 0
    for i in range(L + 1):
        if (c >> i) & 1:
            phi |= 1 << (L - i)
    return phi, L


def poly_mod(a, m):
    dm = m.bit_length() - 1
    while a.bit_length() - 1 >= dm:
        a ^= m << (a.bit_length() - 1 - dm)
    return a


def poly_square(a):
    r, i = 0, 0
    while a:
        if a & 1:
            r |= 1 << (2 * i)
        a >>= 1
        i += 1
    return r


def primitive_by_python(p):
    """Period 2^P - 1 (P = 32 nn - rr prime-exponent): the sequence's
    minimal polynomial has degree P and t^(2^P) = t modulo it."""
    P = 32 * p.nn - p.rr
    x = raw_words(p, 4357, p.nn + 2 * P + 4)
    phi, L = berlekamp_massey([(v >> 31) & 1 for v in x[p.nn:p.nn + 2 * P]])
    if L != P:
        return False
    a = 2
    for _ in range(P):
        a = poly_mod(poly_square(a), phi)
    return a == 2


# ---------------------------------------------------------------- known answers
def test_mt19937_known_answers():
    p = A.mt19937_params()
    assert A.mt_is_primitive(p)
    k = A.mt_equidistribution(p, 32)
    assert k[0] == 19937 and k[1] == 9968
    assert all(v == 623 for v in k[16:])
    assert sum(19937 // v - kv for v, kv in enumerate(k, 1)) == 6750


def test_primitivity_check_agrees_with_python_on_random_twists():
    rng = np.random.default_rng(5)
    base = A.mt_create(521, 0, 1)
    verdicts = []
    for _ in range(24):
        q = capi.MtParams.from_buffer_copy(base)
        q.aaa = 0x80000000 | int(rng.integers(0, 1 << 31))
        lib = A.mt_is_primitive(q)
        assert lib == primitive_by_python(q)
        verdicts.append(lib)
    assert not all(verdicts)  # most random twist vectors are not primitive


# ------------------------------------------------------------- committed files
@pytest.mark.parametrize("path,P,nn,mm,rr", [(MT19937_FILE, 19937, 624, 312, 31),
                                             (MT521_FILE, 521, 17, 8, 23)])
def test_committed_sets_layout(path, P, nn, mm, rr):
    sets = read_sets(path)
    assert len(sets) == 16
    ids = [s.aaa & 0xFFFF for s in sets]
    assert ids == sorted(ids) and len(set(ids)) == 16
    for s in sets:
        assert (s.nn, s.mm, s.rr, s.ww) == (nn, mm, rr, 32) and 32 * s.nn - s.rr == P
        assert s.aaa >> 31 == 1
        assert (s.shift0, s.shiftB, s.shiftC, s.shift1) == (12, 7, 15, 18)
        assert s.umask == (0xFFFFFFFF << rr) & 0xFFFFFFFF and s.lmask == (~s.umask) & 0xFFFFFFFF
    # distinct ids give distinct recurrences
    assert len({s.aaa for s in sets}) == 16


def test_committed_521_sets_primitive_checked_independently():
    for s in read_sets(MT521_FILE):
        assert primitive_by_python(s), hex(s.aaa)


def test_committed_19937_sets_primitive():
    for s in read_sets(MT19937_FILE):
        assert A.mt_is_primitive(s), hex(s.aaa)


def test_committed_19937_sets_equidistribution():
    """The tempering search reaches MT19937's own equidistribution class."""
    for s in read_sets(MT19937_FILE)[:2]:
        k = A.mt_equidistribution(s, 32)
        assert all(v == 623 for v in k[16:]) and k[0] == 19937
        assert sum(19937 // v - kv for v, kv in enumerate(k, 1)) <= 7000


def output_functionals(p, count):
    """Tempered outputs 0..count-1 of the p-dimensional state as linear
    functions: for each output word, 32 ints whose bit i is that output bit
    for the i-th basis state."""
    P = 32 * p.nn - p.rr
    basis = []  # each basis state is nn words; word 0 only its upper bits
    for w in range(p.nn):
        for b in range(32):
            if w == 0 and not ((p.umask >> b) & 1):
                continue
            st = np.zeros(p.nn, np.uint32)
            st[w] = np.uint32(1 << b)
            basis.append(st)
    assert len(basis) == P
    x = np.stack(basis, axis=1).astype(np.uint32)  # (nn, P)
    um, lm, a = np.uint32(p.umask), np.uint32(p.lmask), np.uint32(p.aaa)
    outs = []
    ring = [x[k] for k in range(p.nn)]
    for j in range(count):
        y = (ring[j] & um) | (ring[j + 1] & lm)
        v = ring[j + p.mm] ^ (y >> np.uint32(1)) ^ np.where(y & np.uint32(1), a, np.uint32(0))
        ring.append(v.astype(np.uint32))
        t = v.copy()
        t ^= t >> np.uint32(p.shift0)
        t ^= (t << np.uint32(p.shiftB)) & np.uint32(p.maskB)
        t ^= (t << np.uint32(p.shiftC)) & np.uint32(p.maskC)
        t ^= t >> np.uint32(p.shift1)
        outs.append(t)
    funcs = []
    for t in outs:
        row = []
        for bit in range(31, -1, -1):  # most significant first
            bits = ((t >> np.uint32(bit)) & np.uint32(1)).astype(np.uint8)
            row.append(int.from_bytes(np.packbits(bits[::-1]).tobytes(), "big") >> ((-P) % 8))
        funcs.append(row)
    return funcs, P


def k_by_rank(funcs, P, v):
    """Largest k with the top v bits of k consecutive outputs linearly
    independent (rank k v)."""
    pivots = {}
    k = 0
    for row in funcs:
        for f in row[:v]:
            while f:
                h = f.bit_length() - 1
                if h not in pivots:
                    pivots[h] = f
                    break
                f ^= pivots[h]
            if f == 0:
                return k
        k += 1
        if (k + 1) * v > P:
            return k
    return k


def test_equidistribution_equals_rank_computation():
    s = read_sets(MT521_FILE)[5]
    funcs, P = output_functionals(s, 530)
    lib = A.mt_equidistribution(s, 32)
    for v in range(1, 33):
        assert lib[v - 1] == k_by_rank(funcs, P, v), v


# ------------------------------------------------------------------- creator
def test_creator_reproduces_committed_sets():
    sets = read_sets(MT521_FILE)
    for k in (0, 7):
        ref = sets[k]
        got = A.mt_create(521, ref.aaa & 0xFFFF, 42)
        assert bytes(got) == bytes(ref)


def test_creator_arguments():
    for args in [(520, 0, 1), (521, -1, 1), (521, 65536, 1)]:
        with pytest.raises(capi.ArmaError) as e:
            A.mt_create(*args)
        assert e.value.code == -1
    with pytest.raises(capi.ArmaError):
        A.mt_create(521, 0, 1, w=64)


def test_dcmt_programme_writes_a_readable_file(tmp_path):
    out = tmp_path / "mt.dat"
    r = subprocess.run([sys.executable, "-m", "arma_b200.dcmt", "-n", "3", "-p", "521", "-s", "9",
                        "-o", str(out)], cwd=ROOT, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sets = read_sets(str(out))
    assert [s.aaa & 0xFFFF for s in sets] == [0, 1, 2]
    assert bytes(sets[1]) == bytes(A.mt_create(521, 1, 9))
