"""The oracle's hQuicksort (oracle_hq_sort: RQuick::sort as the reference's
hQuicksort executable runs it), on the CPU, against

  - a hand-derived case whose result needs none of the random bits;
  - a second restatement here in pure Python with its own MT19937-64
    (Matsumoto and Nishimura's published generator, which std::mt19937_64
    is), pinned to the C++ standard's known answer for that generator;
  - the executable's own check (src/executables/HQuicksort.cpp:360-396): the
    PEs' outputs in rank order are the sorted input, every PE's sorted."""
import bisect

import numpy as np
import pytest

from dist_oracle import pack_list
from inputs import random_strings, with_duplicates

HQ_SEED = 3469931


class MT64:
    """MT19937-64 (Matsumoto and Nishimura, 2004): 312 words of state, the
    std::mt19937_64 parameters."""
    NN, MM = 312, 156
    A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF
    M64 = (1 << 64) - 1

    def __init__(self, seed):
        mt = [seed & self.M64]
        for i in range(1, self.NN):
            mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & self.M64)
        self.mt, self.i = mt, self.NN

    def __call__(self):
        mt, NN, MM = self.mt, self.NN, self.MM
        if self.i >= NN:
            for k in range(NN):
                x = (mt[k] & self.UM) | (mt[(k + 1) % NN] & self.LM)
                mt[k] = mt[(k + MM) % NN] ^ (x >> 1) ^ (self.A if x & 1 else 0)
            self.i = 0
        x = mt[self.i]
        self.i += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & self.M64


class Bits:
    """RandomBitStore: one 64-bit draw serves 64 bits, lowest first."""

    def __init__(self, seed):
        self.g, self.left, self.v = MT64(seed), 0, 0

    def next(self):
        if not self.left:
            self.v, self.left = self.g(), 64
        b = self.v & 1
        self.v >>= 1
        self.left -= 1
        return b


def rquick(pes, seed=HQ_SEED):
    """RQuick::sort (sorter/RQuick/RQuick.hpp:834-1104, sortRec :415-627) on
    lists of bytes, one per PE; returns the PEs' sorted lists."""
    p = len(pes)
    pes = [list(v) for v in pes]
    pw = 1
    while pw * 2 <= p:
        pw *= 2
    for q in range(pw, p):
        pes[q - pw] += pes[q]
        pes[q] = []
    pes = [sorted(v) for v in pes]
    bits = [Bits(seed + q) for q in range(pw)]
    P = pw
    while P >= 2:
        for b in range(0, pw, P):
            beg = {}
            for q in range(b, b + P):
                c = len(pes[q])
                beg[q] = (c - 2) // 2 + (bits[q].next() if c % 2 else 0) if c > 2 else 0
            m = min(len(pes[b]), 2)
            piv = pes[b][beg[b] + (bits[b].next() if m == 2 else 0)] if m else b""
            sep = {}
            for q in range(b, b + P):
                v = pes[q]
                lo = bisect.bisect_left(v, piv)
                hi = bisect.bisect_right(v, piv)
                opt = len(v) // 2 + (bits[q].next() if len(v) % 2 else 0)
                sep[q] = min(opt, hi) if lo < opt else lo
            nxt = {}
            for q in range(b, b + P):
                r = b + (q - b + P // 2) % P
                if q - b < P // 2:
                    nxt[q] = sorted(pes[q][:sep[q]] + pes[r][:sep[r]])
                else:
                    nxt[q] = sorted(pes[q][sep[q]:] + pes[r][sep[r]:])
            for q in range(b, b + P):
                pes[q] = nxt[q]
        P //= 2
    return pes


def oracle_pes(orc, pes, seed=HQ_SEED):
    strs = [s for v in pes for s in v]
    chars, offs, lens, _ = pack_list(strs)
    s = orc.Strings(chars, offs.astype(np.uint64), lens.astype(np.uint32))
    pb = np.concatenate([[0], np.cumsum([len(v) for v in pes])]).astype(np.uint64)
    o = orc.hq_sort(s, pb, seed)
    out, k = [], 0
    for c in o["counts"].astype(np.int64):
        out.append([strs[int(i)] for i in o["source"][k:k + c]])
        k += c
    return out


def test_mt19937_64_known_answer():
    """The C++ standard ([rand.predef]): the 10000th draw of a default-seeded
    (5489) mt19937_64 is 9981545732273789042."""
    g = MT64(5489)
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


def test_hand_case(orc):
    """p = 2.  PE 0's two middle strings are both "m", so the pivot is "m"
    whatever bit picks it; both PEs hold 4 strings (no bits in the split).
    PE 0: lower_bound 1, upper_bound 3, middle 2 -> keeps a m, sends m z.
    PE 1: lower_bound = upper_bound = 2 = middle -> keeps n y, sends b c."""
    pes = [[b"z", b"m", b"a", b"m"], [b"y", b"b", b"n", b"c"]]
    want = [[b"a", b"b", b"c", b"m"], [b"m", b"n", b"y", b"z"]]
    assert rquick(pes) == want
    assert oracle_pes(orc, pes) == want


def split_evenly(strs, p, rng):
    cuts = np.sort(rng.integers(0, len(strs) + 1, p - 1)) if p > 1 else np.zeros(0, np.int64)
    b = [0] + cuts.tolist() + [len(strs)]
    return [strs[b[q]:b[q + 1]] for q in range(p)]


CASES = [
    ("random", lambda: random_strings(700, 0, 12, b"ABCD", seed=71)),
    ("dups", lambda: with_duplicates(random_strings(600, 0, 6, b"AB", seed=72), 0.5, seed=73)),
    ("equal", lambda: [b"same"] * 300 + [b""] * 40),
    ("empties", lambda: [b""] * 50 + random_strings(200, 1, 4, b"xy", seed=74)),
]


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 7, 8, 16])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_restatement(orc, name, make, p):
    strs = make()
    rng = np.random.default_rng(p * 31 + len(name))
    pes = split_evenly(strs, p, rng)
    got = oracle_pes(orc, pes)
    assert got == rquick(pes)
    # the executable's check: rank order is the sorted input, each PE sorted
    assert [s for v in got for s in v] == sorted(strs)
    assert len(got) == p


@pytest.mark.parametrize("pes", [
    [[], [b"b", b"a"]],                 # the subcube's first PE is empty: the pivot is ""
    [[], [], [b"", b"c"], [b"a"]],
    [[b""] * 3, [b""] * 5],
    [[], []],
    [[b"one"]],
])
def test_oracle_edges(orc, pes):
    got = oracle_pes(orc, pes)
    assert got == rquick(pes)
    assert [s for v in got for s in v] == sorted(s for v in pes for s in v)


def test_seed_changes_split(orc):
    """Ties split by the random bits: other seeds give other counts."""
    pes = [[b"x"] * 5, [b"x"] * 3]
    seen = {tuple(len(v) for v in oracle_pes(orc, pes, seed)) for seed in range(HQ_SEED, HQ_SEED + 40)}
    for seed in (HQ_SEED, HQ_SEED + 7):
        assert oracle_pes(orc, pes, seed) == rquick(pes, seed)
    assert len(seen) > 1 and all(sum(c) == 8 for c in seen)


def test_oracle_matches_restatement_random_layouts(orc):
    """Random PE layouts (empty PEs, few distinct strings, 1-12 PEs, random
    seeds): the oracle and the pure-Python restatement agree exactly."""
    from hypothesis import given, settings, strategies as st

    word = st.binary(min_size=0, max_size=5).map(lambda b: bytes(65 + (x % 3) for x in b))

    @settings(max_examples=150, deadline=None, derandomize=True)
    @given(st.lists(st.lists(word, max_size=12), min_size=1, max_size=12), st.integers(0, 1 << 30))
    def check(pes, seed):
        assert oracle_pes(orc, pes, seed) == rquick(pes, seed)

    check()
