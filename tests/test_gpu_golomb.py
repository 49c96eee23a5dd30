"""Golomb/delta coding on the GPU (dsss_golomb_encode / dsss_golomb_decode):
the words equal the oracle's restatement of the reference's coder (itself
pinned to the reference's compiled getDeltaEncoding, test_oracle_pins.py),
word for word, and read back to the values; blocks much longer than one
decoding chunk, codes whose unary part spans several words, parameters that
are not powers of two and empty ranges included; malformed input is
rejected."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint64)


def roundtrip(dsss, orc, ctx, values, counts, bs):
    want, want_rw = orc.golomb_encode(values, counts, bs)
    words, rw = dsss.golomb_encode(ctx, dev(values), counts, bs)
    assert np.array_equal(host(words), want)
    assert rw.tolist() == want_rw.tolist()
    got, bc = dsss.golomb_decode(ctx, words)
    assert np.array_equal(host(got), np.asarray(values, np.uint64))
    assert bc.tolist() == [c for c in counts if c]


def test_golden_blocks(dsss, orc, ctx):
    with open(os.path.join(GOLDEN, "golomb_ref.json")) as f:
        g = json.load(f)
    for blk in g["blocks"]:
        v = np.array([int(x) for x in blk["values"]], np.uint64)
        want = np.array([int(x) for x in blk["words"]], np.uint64)
        words, rw = dsss.golomb_encode(ctx, dev(v), [len(v)], [blk["b"]])
        assert np.array_equal(host(words), want)
        got, bc = dsss.golomb_decode(ctx, dev(want))
        assert np.array_equal(host(got), v) and bc.tolist() == [len(v)]
    for m, c, b in g["params"]:
        assert dsss.golomb_param(int(m), int(c)) == int(b)


@pytest.mark.parametrize("seed", range(6))
def test_hash_exchange_blocks(dsss, orc, ctx, seed):
    """p destinations of sorted 64-bit hashes with the exchange's b, some
    destinations empty, up to 40k hashes per block (hundreds of chunks)."""
    rng = np.random.default_rng(seed)
    p = [3, 8, 16, 5, 64, 2][seed]
    counts = [int(x) for x in rng.integers(0, 40000, p)]
    counts[int(rng.integers(0, p))] = 0
    vals = np.concatenate([np.sort(rng.integers(0, 2**64 - 1, c, dtype=np.uint64)) for c in counts])
    bs = [dsss.golomb_param_hashes(c, p) for c in counts]
    assert bs == [orc.golomb_param_hashes(c, p) for c in counts]
    roundtrip(dsss, orc, ctx, vals, counts, bs)


@pytest.mark.parametrize("b", [3, 5, 7, 8, 1000, 20000000000])
def test_small_gaps_any_b(dsss, orc, ctx, b):
    rng = np.random.default_rng(b % 97)
    counts = [1, 0, 2500, 1, 7, 12000]
    vals = np.concatenate([np.cumsum(rng.integers(0, 60, c)).astype(np.uint64) for c in counts])
    roundtrip(dsss, orc, ctx, vals, counts, [b] * len(counts))


def test_long_unary_parts(dsss, orc, ctx):
    """Gaps of thousands of b: unary runs over several words and chunks."""
    rng = np.random.default_rng(5)
    v = np.cumsum(rng.integers(0, 3, 3000)).astype(np.uint64)
    v[1000:] += np.uint64(8 * 5000)
    v[2000:] += np.uint64(8 * 70000)
    roundtrip(dsss, orc, ctx, v, [len(v)], [8])


def test_duplicate_positions(dsss, orc, ctx):
    """The duplicate answers' form: positions plus offsets, b = max(getB, 8)."""
    rng = np.random.default_rng(9)
    counts, vals, bs = [], [], []
    off = 0
    for r in range(7):
        m = int(rng.integers(0, 5000))
        c = int(rng.integers(0, m + 1)) if m else 0
        pos = np.sort(rng.choice(m, c, replace=False)).astype(np.uint64) + np.uint64(off) if c else np.zeros(0, np.uint64)
        off += m
        counts.append(c)
        vals.append(pos)
        bs.append(max(8, dsss.golomb_param(m, c)))
    roundtrip(dsss, orc, ctx, np.concatenate(vals), counts, bs)


def test_exact_word_ends_and_single_values(dsss, orc, ctx):
    """Blocks whose codes end on a word boundary (no padding) and blocks of
    one value (no bit words)."""
    # b = 2^31: every gap below b codes to 1 + 31 bits, two codes per word
    v = np.array([5, 6, 7, 8, 9], np.uint64)
    roundtrip(dsss, orc, ctx, v, [5], [1 << 31])
    roundtrip(dsss, orc, ctx, np.array([42, 7, 2**64 - 1], np.uint64), [1, 1, 1], [8, 8, 8])


def test_rejects(dsss, ctx):
    import ctypes
    with pytest.raises(dsss.DsssError):
        dsss.golomb_encode(ctx, dev(np.array([5, 3], np.uint64)), [2], [8])  # descending
    with pytest.raises(dsss.DsssError):
        dsss.golomb_encode(ctx, dev(np.array([1, 2], np.uint64)), [2], [0])  # b = 0
    with pytest.raises(dsss.DsssError):
        dsss.golomb_decode(ctx, dev(np.array([9, 8, 1], np.uint64)))  # S past the buffer
    words, _ = dsss.golomb_encode(ctx, dev(np.arange(10, dtype=np.uint64)), [4, 6], [8, 8])
    with pytest.raises(dsss.DsssError):
        dsss.golomb_decode(ctx, words, max_blocks=1)
    n = ctypes.c_uint64(0)
    nb = ctypes.c_uint32(0)
    assert dsss.lib().dsss_golomb_decode(ctx.h, None, 0, None, 0, ctypes.byref(n), None, 0, ctypes.byref(nb),
                                         None) == 0 and n.value == 0
