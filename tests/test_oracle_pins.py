"""The oracle pinned to the reference: golden fixtures made from the reference's
own code (tests/golden/make_golden.py), the reference's PD-exchange
known-answer test, and — where oracle/_ref is built — direct comparisons with
the reference's compiled pieces on more inputs.  CPU only."""
import json
import os

import numpy as np
import pytest

from inputs import cases, long_prefix, random_strings, with_duplicates

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def strings_of(orc, strs):
    lens = np.array([len(x) for x in strs], np.uint32)
    offs = np.zeros(len(strs), np.uint64)
    if strs:
        offs[1:] = np.cumsum(lens.astype(np.uint64) + 1)[:-1]
    chars = np.frombuffer(b"".join(x + b"\0" for x in strs) + b"\0" * 32, np.uint8).copy()
    return orc.Strings(chars, offs, lens)


def test_xxh64_golden(orc):
    for v in load("xxh64_ref.json"):
        assert format(orc.xxh64(bytes.fromhex(v["data"])), "016x") == v["xxh64"]
    # published test vector of XXH64 used as a probe of the reference port
    assert orc.xxh64(b"HELLOWOR") == 0x27DB29BA10CD21C3


def test_xxh64_len32_is_the_ports_variant(orc):
    """The reference port merges the four lanes only for length > 32
    (hash/xxhash.hpp:608); its 32-byte hash is the one in the golden file."""
    v = [x for x in load("xxh64_ref.json") if len(x["data"]) == 64][0]
    assert format(orc.xxh64(bytes.fromhex(v["data"])), "016x") == v["xxh64"]


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
def test_xxh64_vs_reference_code(orc):
    rng = np.random.default_rng(5)
    for L in list(range(0, 200)) + [1000, 4096]:
        d = bytes(rng.integers(0, 256, L).astype(np.uint8))
        assert orc.xxh64(d) == orc.ref_xxh64(d)


def test_dp_golden(orc):
    for name, v in load("dp_ref.json").items():
        strs = [bytes.fromhex(x) for x in v["strings"]]
        s = strings_of(orc, strs)
        pb = np.array([0, len(strs)], np.uint64)
        order, lcp = orc.local_sort(s, pb)
        # byte-identical strings may sit in any order; compare the strings
        assert [strs[i] for i in order] == [strs[i] for i in v["order"]], name
        assert lcp.tolist() == v["lcp"], name
        dp, _ = orc.dp_rounds(s, pb, order, lcp)
        assert dp.tolist() == v["dp"], name


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,strs", cases())
def test_local_sort_vs_radixsort_ci3(orc, name, strs):
    s = strings_of(orc, strs)
    order, lcp = orc.local_sort(s, np.array([0, len(strs)], np.uint64))
    ro, rl = orc.ref_local_sort(strs)
    assert [strs[i] for i in order] == [strs[i] for i in ro]
    assert lcp.tolist() == rl.tolist()


@pytest.mark.skipif(not __import__("oracle").ref_dp_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,strs", cases())
def test_dp_vs_reference_bloomfilter(orc, name, strs):
    """computeDistinguishingPrefixes of the reference (one PE) vs the oracle's
    rounds over one PE and over several simulated PEs."""
    if not strs:
        return
    ro, rl, rdp = orc.ref_dp_single_pe(strs)
    s = strings_of(orc, strs)
    n = len(strs)
    pb1 = np.array([0, n], np.uint64)
    order, lcp = orc.local_sort(s, pb1)
    dp, _ = orc.dp_rounds(s, pb1, order, lcp)
    assert dp.tolist() == rdp.tolist()
    by_string = {}
    for i, x in zip(order, dp):
        by_string.setdefault(strs[i], set()).add(int(x))
    for p in (2, 3, 7):
        pb = np.array([q * n // p for q in range(p + 1)], np.uint64)
        o2, l2 = orc.local_sort(s, pb)
        d2, _ = orc.dp_rounds(s, pb, o2, l2)
        for i, x in zip(o2, d2):
            assert int(x) in by_string[strs[i]], (p, strs[i])


def test_dp_rounds_schedule(orc):
    """Depths 8, 24, 40, 72, 136, 264, 520, 1032 (prefix_doubling.hpp:162,181-193):
    strings sharing 600 bytes end at EOS in the round of depth 1032."""
    strs = long_prefix(200, 600, 20, 9)
    s = strings_of(orc, strs)
    pb = np.array([0, len(strs)], np.uint64)
    order, lcp = orc.local_sort(s, pb)
    dp, counts = orc.dp_rounds(s, pb, order, lcp)
    assert len(counts) == 8 and counts[-1] == 0
    assert all(int(d) == len(strs[i]) for i, d in zip(order, dp))


def test_merge_golden(orc):
    for name, v in load("merge_ref.json").items():
        for pe in v["pes"]:
            chars = np.frombuffer(bytes.fromhex(pe["chars"]), np.uint8)
            idx, src, mlcp, old = orc.merge(chars, pe["lcp"], pe["counts"], pe["offsets"])
            assert idx.tolist() == pe["index"], name
            assert src.tolist() == pe["pe"], name
            assert mlcp.tolist() == pe["merged_lcp"], name
            assert old.tolist() == pe["old_lcp"], name


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("p", [2, 3, 4, 8])
def test_merge_vs_reference_losertree(orc, p):
    strs = with_duplicates(random_strings(1500, 0, 16, b"ABC", 40 + p), 0.4, 41)
    s = strings_of(orc, strs)
    n = len(strs)
    pb = np.array([q * n // p for q in range(p + 1)], np.uint64)
    order, lcp = orc.local_sort(s, pb)
    dp, _ = orc.dp_rounds(s, pb, order, lcp)
    iv = orc.partition(s, pb, order, dp)
    ex = orc.exchange(s, pb, order, lcp, dp, iv)
    start = 0
    for r in range(p):
        cnt = int(ex["counts"][r].sum())
        cb, ce = int(ex["char_begin"][r]), int(ex["char_begin"][r + 1])
        lc = ex["lcp"][start:start + cnt]
        a = orc.merge(ex["chars"][cb:ce], lc, ex["counts"][r], ex["offsets"][r])
        b = orc.ref_lcp_merge(ex["chars"][cb:ce], lc, ex["counts"][r], ex["offsets"][r])
        for x, y in zip(a, b):
            assert x.tolist() == y.tolist()
        start += cnt


def test_pd_exchange_kat(orc):
    """src/tests/alltoallStrings_tests.cpp:129-163 (AllToAllStringImplPrefixDoubling)."""
    for case in load("pd_exchange_kat.json"):
        p = case["p"]
        strs, lcps, dps, sends = [], [], [], []
        for pe in case["pes"]:
            strs += [bytes.fromhex(x) for x in pe["strings"]]
            lcps += pe["lcp"]
            dps += pe["dp"]
            sends.append(pe["send"])
        s = strings_of(orc, strs)
        n = len(strs)
        per = n // p
        pb = np.array([q * per for q in range(p + 1)], np.uint64)
        order = np.arange(n, dtype=np.uint64)
        ex = orc.exchange(s, pb, order, np.array(lcps, np.uint64), np.array(dps, np.uint64),
                          np.array(sends, np.uint64))
        # every PE receives the same bytes and LCPs (the test checks each rank)
        m = len(case["expected_lcp"])
        for r in range(p):
            cb, ce = int(ex["char_begin"][r]), int(ex["char_begin"][r + 1])
            assert ex["chars"][cb:ce].tobytes().hex() == case["expected_raw"], (p, r, case["simulate_duplicates"])
            assert ex["lcp"][r * m:(r + 1) * m].tolist() == case["expected_lcp"], (p, r, case["simulate_duplicates"])


@pytest.mark.parametrize("p", [1, 2, 3, 5, 8])
def test_pd_sort_oracle_global_order(orc, dsss, p):
    """The concatenated merged outputs are the globally sorted strings (the
    reference's --check, mpi/is_sorted.hpp:106-199), and DP >= the exact DP."""
    hs = dsss.gen_dn(3000, 60, 30, seed=p)
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(hs.n, p)
    r = orc.pd_sort(s, pb)
    if p == 1:
        assert r["recv_counts"].tolist() == [0]
        return
    local = [[int(r["order"][int(pb[q]) + i]) for i in range(int(pb[q + 1] - pb[q]))] for q in range(p)]
    merged = [s.get(local[int(q)][int(i)]) for i, q in zip(r["perm_index"], r["perm_pe"])]
    assert merged == sorted(s.get(i) for i in range(hs.n))
    assert sorted(zip(r["perm_pe"].tolist(), r["perm_index"].tolist())) == \
        sorted((q, i) for q in range(p) for i in range(len(local[q])))


def test_varint_reference_known_answer(orc):
    """The reference's own test (src/tests/integerCompression_tests.cpp:11-60):
    1, 2^8, 2^16, ..., 2^56 written twice as two ranges take 37 bytes each,
    and read back unchanged."""
    nums = [1 << (8 * i) for i in range(8)]
    data, per = orc.varint_encode(nums + nums, [8, 8])
    assert per.tolist() == [37, 37]
    assert orc.varint_decode(data, 16).tolist() == nums + nums
    # LEB128 bytes of single values (7 bits per byte, low first, high bit = more)
    assert orc.varint_encode([300], [1])[0].tobytes() == b"\xac\x02"
    assert orc.varint_encode([2**32 - 1], [1])[0].tobytes() == b"\xff\xff\xff\xff\x0f"


def _golomb_fixture():
    with open(os.path.join(GOLDEN, "golomb_ref.json")) as f:
        return json.load(f)


def test_golomb_golden(orc):
    """The oracle's Golomb/delta coder writes, block for block, the words the
    reference's coder wrote (getDeltaEncoding over thrill's bit streams,
    framed as AllToAllHashesGolomb frames a destination's hashes), and reads
    them back; getB agrees on every pair."""
    g = _golomb_fixture()
    for blk in g["blocks"]:
        v = np.array([int(x) for x in blk["values"]], np.uint64)
        want = np.array([int(x) for x in blk["words"]], np.uint64)
        got, rw = orc.golomb_encode(v, [len(v)], [blk["b"]])
        assert np.array_equal(got, want)
        assert int(rw[0]) == len(want)
        dec, counts = orc.golomb_decode(want)
        assert np.array_equal(dec, v) and counts.tolist() == [len(v)]
    for m, c, b in g["params"]:
        assert orc.golomb_param(int(m), int(c)) == int(b)


def test_golomb_blocks_back_to_back(orc):
    """Several destinations in one buffer, empty ones taking no words, as the
    exchange sends them; the receiver reads block after block."""
    rng = np.random.default_rng(3)
    counts = [5, 0, 1, 40, 0, 0, 17]
    vals = np.concatenate([np.sort(rng.integers(0, 2**64 - 1, c, dtype=np.uint64)) for c in counts])
    bs = [orc.golomb_param_hashes(c, len(counts)) for c in counts]
    words, rw = orc.golomb_encode(vals, counts, bs)
    assert [int(x) == 0 for x in rw] == [c == 0 for c in counts]
    dec, bc = orc.golomb_decode(words)
    assert np.array_equal(dec, vals)
    assert bc.tolist() == [c for c in counts if c]


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="oracle/_ref not built")
def test_golomb_vs_reference_coder(orc):
    """Random sorted blocks (64-bit hashes, offsets, small gaps, b a power of
    two or not): the oracle's words equal the reference coder's and both read
    back to the values."""
    rng = np.random.default_rng(11)
    for trial in range(120):
        c = int(rng.integers(1, 200))
        mode = trial % 3
        if mode == 0:
            v = np.sort(rng.integers(0, 2**64 - 1, c, dtype=np.uint64))
            choices = [orc.golomb_param_hashes(c, 8), 1 << 54]
        elif mode == 1:
            v = np.sort(rng.integers(0, 10**6, c, dtype=np.uint64))
            choices = [8, 16, 3, 5, 1000, 20000000000, max(8, orc.golomb_param(10**6, c))]
        else:
            v = np.cumsum(rng.integers(0, 9, c)).astype(np.uint64)
            choices = [3, 7, 8, 64]
        for b in choices:
            want = orc.ref_golomb_block(v, b)
            got, _ = orc.golomb_encode(v, [c], [b])
            assert np.array_equal(got, want), (trial, b)
            assert np.array_equal(orc.ref_golomb_unblock(want, c + 4), v)
