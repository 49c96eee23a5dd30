"""Tuning knobs change how the path runs, never its results: the fingerprint
filter of the distinguishing-prefix rounds (forced on for small inputs), the
pivot passes of the string sort (off), the small-segment cutoff, and the
hash rounds split into hashing and insert kernels."""
import numpy as np
import pytest

from inputs import cases
from test_gpu_parity import check_pd, host_of, u64

pytestmark = pytest.mark.gpu

CASES = [c for c in cases() if len(c[1]) >= 8]
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("p", [2, 5])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_filter_forced(dsss, orc, ctx, name, strs, p):
    hs = host_of(dsss, strs)
    with dsss.tuned(dp_filter_min=0):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p)
    check_pd(dsss, orc, hs, out, p)


@pytest.mark.parametrize("bits", [4, 64])
def test_filter_bits(dsss, orc, ctx, bits):
    """Few filter bits per key: many candidates (every one checked exactly)."""
    hs = dsss.gen_suffix_strings(60000, 256, seed=3)
    with dsss.tuned(dp_filter_min=0, dp_filter_bits=bits):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 4)
    check_pd(dsss, orc, hs, out, 4)


def test_filter_batched(dsss, ctx):
    """Per-set filter regions: a batch with repeated sets gives each set its
    single-set result."""
    h1 = dsss.gen_dn(20000, 100, 50, seed=31)
    h2 = dsss.gen_suffix_strings(30000, 256, seed=4)
    hs, sb = dsss.concat_sets([h1, h2, h1, h2])
    pb = dsss.batched_parts(sb, 4)
    with dsss.tuned(dp_filter_min=0):
        out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), 4, 4, pb)
    for s, h in enumerate([h1, h2, h1, h2]):
        ref = dsss.pd_sort(ctx, dsss.DeviceStrings(h), 4)
        b, e = int(sb[s]), int(sb[s + 1])
        assert np.array_equal(u64(out["dp"], hs.n)[b:e], u64(ref["dp"], h.n)), s
        assert np.array_equal(u64(out["perm_index"], hs.n)[b:e], u64(ref["perm_index"], h.n)), s


@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_dp_split(dsss, orc, ctx, name, strs):
    """Hash rounds as separate hashing and insert kernels: the oracle's result."""
    hs = host_of(dsss, strs)
    with dsss.tuned(dp_split=1):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 3)
    check_pd(dsss, orc, hs, out, 3)


def test_dp_split_batched(dsss, ctx):
    """Split hash rounds over per-set table regions: each set's own result."""
    h1 = dsss.gen_dn(20000, 100, 50, seed=33)
    h2 = dsss.gen_suffix_strings(30000, 256, seed=5)
    hs, sb = dsss.concat_sets([h1, h2, h1])
    pb = dsss.batched_parts(sb, 4)
    with dsss.tuned(dp_split=1):
        out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), 3, 4, pb)
    for s, h in enumerate([h1, h2, h1]):
        ref = dsss.pd_sort(ctx, dsss.DeviceStrings(h), 4)
        b, e = int(sb[s]), int(sb[s + 1])
        assert np.array_equal(u64(out["dp"], hs.n)[b:e], u64(ref["dp"], h.n)), s
        assert np.array_equal(u64(out["perm_index"], hs.n)[b:e], u64(ref["perm_index"], h.n)), s


@pytest.mark.parametrize("knobs", [dict(sort_pivot=0), dict(sort_small_max=64), dict(sort_small_max=2, sort_pivot=0),
                                   dict(sort_graph_max_n=0), dict(sort_graph_max_n=0, sort_small_max=64)])
def test_sort_knobs(dsss, orc, ctx, knobs):
    hs = dsss.gen_suffix_strings(50000, 256, seed=6)
    n = hs.n
    with dsss.tuned(**knobs):
        order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), 1)
    ro, rl = orc.local_sort(orc.Strings.from_host(hs), np.array([0, n], np.uint64))
    assert np.array_equal(u64(order, n), ro)
    assert np.array_equal(u64(lcp, n), rl)


def test_autotune_picks_a_grid_setting(dsss, orc, ctx):
    """dsss_autotune leaves one setting of its grid in force; results stay exact."""
    hs = dsss.gen_suffix_strings(80000, 256, seed=8)
    ds = dsss.DeviceStrings(hs)
    with dsss.tuned(sort_small_max=-1, sort_pivot=-1, sort_split_min=-1, sort_bits=-1, sort_seg_bits=-1):
        t = dsss.autotune(ctx, ds, 4, trials=1)
        assert t["settings_tried"] == 30
        assert t["sort_small_max"] in (256, 1024, 4096) and t["sort_pivot"] in (0, 1)
        assert (t["sort_split_min"], t["sort_bits"], t["sort_seg_bits"]) in ((0, 0, 0), (65536, 0, 0), (0, 2, 0),
                                                                             (0, 0, 1), (0, 3, 1))
        assert dsss.tune_get("sort_seg_bits") == t["sort_seg_bits"]
        assert dsss.tune_get("sort_split_min") == t["sort_split_min"]
        assert dsss.tune_get("sort_bits") == t["sort_bits"]
        assert 0 < t["best_ms"] <= t["default_ms"]
        assert dsss.tune_get("sort_small_max") == t["sort_small_max"]
        out = dsss.pd_sort(ctx, ds, 4)
        check_pd(dsss, orc, hs, out, 4)


@pytest.mark.parametrize("graph", [0, 1 << 22])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_sort_host_loop_and_graph(dsss, orc, ctx, name, strs, graph):
    """The MSD passes driven from the host (one read-back per pass) and as one
    CUDA graph with a device-side loop condition give the same order and LCPs."""
    hs = host_of(dsss, strs)
    n = hs.n
    with dsss.tuned(sort_graph_max_n=graph, sort_small_max=32):
        order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), 3 if n >= 3 else 1)
    pb = dsss.equal_parts(n, 3 if n >= 3 else 1)
    ro, rl = orc.local_sort(orc.Strings.from_host(hs), pb)
    assert np.array_equal(u64(order, n), ro)
    assert np.array_equal(u64(lcp, n), rl)


@pytest.mark.parametrize("early", [None, 1, 4999])
def test_prefix_speculation(dsss, orc, ctx, early):
    """The string sort guesses a segment's common prefix from 256 evenly
    spaced members and writes the keys at that depth in the same pass; the
    guess holds (early=None) or one member that the sample misses leaves the
    shared head early (positions 1 and 4999 of 10000), and the sort falls back
    to the exact depth.  Order and LCPs equal the oracle's either way."""
    rng = np.random.default_rng(11)
    head = b"XY" * 10
    strs = [head + bytes(rng.integers(65, 91, size=int(rng.integers(0, 30)), dtype=np.uint8)) for _ in range(10000)]
    if early is not None:
        strs[early] = head[:5] + b"A" + strs[early][6:]
    hs = host_of(dsss, strs)
    n = hs.n
    for p in (1, 3):
        pb = np.linspace(0, n, p + 1).astype(np.uint64)
        for small in (0, 64):  # 64: every segment above 64 strings takes the MSD passes
            order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), p, part_begin=pb, small_sort_max=small)
            ro, rl = orc.local_sort(orc.Strings.from_host(hs), pb)
            assert np.array_equal(u64(order, n), ro)
            assert np.array_equal(u64(lcp, n), rl)


@pytest.mark.parametrize("w", [8, 16])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_copy_word(dsss, orc, ctx, name, strs, w):
    """Output strings copied with 8- or 16-byte stores: the merge-sort path
    and hQuicksort give the oracle's bytes either way."""
    from test_gpu_hq import check_hq
    from test_gpu_ms import check_ms
    hs = host_of(dsss, strs)
    pb = np.linspace(0, hs.n, 4).astype(np.uint64)
    with dsss.tuned(copy_word=w):
        ms = dsss.ms_sort(ctx, dsss.DeviceStrings(hs), 3, part_begin=pb)
        hq = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), 3, part_begin=pb)
    check_ms(dsss, orc, hs, ms, pb)
    check_hq(dsss, orc, hs, hq, pb)


@pytest.mark.parametrize("w", [8, 16])
def test_copy_word_lengths(dsss, orc, ctx, w):
    """Every length from 0 to 80 at every alignment of the output: heads,
    tails and strings shorter than one store word."""
    from test_gpu_hq import check_hq
    rng = np.random.default_rng(9)
    strs = [bytes(rng.integers(65, 91, int(k)).astype(np.uint8)) for k in rng.integers(0, 81, 3000)]
    hs = host_of(dsss, strs)
    pb = np.array([0, 1000, 3000], np.uint64)
    with dsss.tuned(copy_word=w):
        hq = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), 2, part_begin=pb)
    check_hq(dsss, orc, hs, hq, pb)


@pytest.mark.parametrize("share", [0, 1, 64])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_dp_digest(dsss, orc, ctx, name, strs, share):
    """Dense hash rounds with the prefixes hashed in arena order (share 64:
    nearly every round; 1: only rounds where every position hashes; 0: off):
    the oracle's result."""
    hs = host_of(dsss, strs)
    with dsss.tuned(dp_digest=share):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 3)
    check_pd(dsss, orc, hs, out, 3)


def test_dp_digest_batched(dsss, ctx):
    """Arena-order hashes over per-set table regions: each set's own result."""
    h1 = dsss.gen_dn(20000, 100, 50, seed=35)
    h2 = dsss.gen_suffix_strings(30000, 256, seed=7)
    hs, sb = dsss.concat_sets([h1, h2, h1])
    pb = dsss.batched_parts(sb, 4)
    with dsss.tuned(dp_digest=64):
        out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), 3, 4, pb)
    with dsss.tuned(dp_digest=0):
        for s, h in enumerate([h1, h2, h1]):
            ref = dsss.pd_sort(ctx, dsss.DeviceStrings(h), 4)
            b, e = int(sb[s]), int(sb[s + 1])
            assert np.array_equal(u64(out["dp"], hs.n)[b:e], u64(ref["dp"], h.n)), s
            assert np.array_equal(u64(out["perm_index"], hs.n)[b:e], u64(ref["perm_index"], h.n)), s


@pytest.mark.parametrize("share", [0, 1, 64])
@pytest.mark.parametrize("p", [3, 16])
def test_dp_digest_per_pe_orders(dsss, orc, ctx, share, p):
    """The distinguishing-prefix stage on per-PE local orders, where equal
    prefixes on different PEs are separate roots whose hashes meet in the
    table: the arena-order form (share 1 / 64) finds the same duplicates
    (shared slots, their owners, the kind-2 strings kept) as the sorted-order
    form (share 0) and the oracle."""
    import torch
    from inputs import long_prefix, random_strings, with_duplicates
    strs = with_duplicates(long_prefix(3000, 90, 12, 71) + random_strings(3000, 0, 40, b"AB", 72), 0.3, 73)
    hs = host_of(dsss, strs)
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(hs.n, p)
    ro, rl = orc.local_sort(s, pb)
    rdp, rcounts = orc.dp_rounds(s, pb, ro, rl)
    ds = dsss.DeviceStrings(hs)
    order = torch.from_numpy(ro.astype(np.int32)).cuda()
    lcp = torch.from_numpy(rl.astype(np.int32)).cuda()
    with dsss.tuned(dp_digest=share):
        dp, counts = dsss.dp_prefixes(ctx, ds, order, lcp, p)
    assert np.array_equal(u64(dp, hs.n), rdp)
    assert counts.tolist() == rcounts.tolist()


def _depth_families():
    """Inputs whose dense hash round falls at each of the depths the string
    sort's first pass hashes (8, 24, 40, 72), with lengths around each."""
    rng = np.random.default_rng(77)
    fams = []
    for common in (0, 12, 30, 60):
        strs = []
        for k in range(4000):
            L = int(rng.choice([common + 3, common + 8, common + 20, 7, 8, 9, 23, 24, 25, 39, 40, 41, 71, 72, 73,
                                100, 200]))
            body = bytes(rng.integers(65, 91, L).astype(np.uint8))
            strs.append((b"Q" * common + body)[:max(L, 1)])
        fams.append(strs)
    return fams


@pytest.mark.parametrize("fam", range(4), ids=["dense8", "dense24", "dense40", "dense72"])
def test_root_digests_checked(dsss, orc, ctx, fam):
    """The prefix hashes stored by the string sort's first pass equal XXH64 of
    the prefix at every depth where a dense round reads them (dp_check
    recomputes each one and fails the call on a mismatch), and the result is
    the oracle's."""
    hs = host_of(dsss, _depth_families()[fam])
    with dsss.tuned(dp_check=1, dp_digest=64):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 3)
    check_pd(dsss, orc, hs, out, 3)
    with dsss.tuned(dp_check=1, dp_digest=64):
        out = dsss.pd_sort(ctx, dsss.gen_dn_device(ctx, 60000, 200, 50, seed=5), 4)
    assert (out["dp"][:60000] == 72).all()


def _split_inputs():
    """String families for the sampled-splitter passes, 60-80k strings each."""
    rng = np.random.default_rng(21)
    letters = [bytes(rng.integers(65, 91, int(k)).astype(np.uint8)) for k in rng.integers(0, 40, 80000)]
    dna = [bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), int(k))) for k in rng.integers(1, 60, 80000)]
    # keys of all-0xFF bytes (the splitter table's padding value) next to 0xFE ones
    ff = [bytes([255]) * int(k) + bytes(rng.integers(254, 256, int(j)).astype(np.uint8))
          for k, j in zip(rng.integers(0, 20, 60000), rng.integers(0, 12, 60000))]
    base = [bytes(rng.integers(97, 100, 12).astype(np.uint8)) for _ in range(5)]
    frequent = [base[int(rng.integers(0, 5))] if rng.random() < 0.9 else
                bytes(rng.integers(97, 123, int(rng.integers(1, 16))).astype(np.uint8)) for _ in range(70000)]
    prefixes = [b"P" * int(k) for k in rng.integers(0, 600, 70000)]
    anybyte = [bytes(rng.integers(1, 256, int(k)).astype(np.uint8)) for k in rng.integers(0, 24, 70000)]
    return [("letters", letters), ("dna", dna), ("ff", ff), ("frequent", frequent), ("prefixes", prefixes),
            ("anybyte", anybyte)]


@pytest.mark.parametrize("small", [0, 64])
@pytest.mark.parametrize("split_min", [0, 4096])
@pytest.mark.parametrize("name,strs", _split_inputs(), ids=[c[0] for c in _split_inputs()])
def test_sort_split(dsss, orc, ctx, name, strs, split_min, small):
    """Large segments split by sampled splitters (sort_split_min 4096: every
    segment from 4096 strings whose next key byte takes few values) or by key
    bytes only (0): the oracle's order and LCPs, in one segment and in three."""
    hs = host_of(dsss, strs)
    n = hs.n
    for p in (1, 3):
        pb = np.linspace(0, n, p + 1).astype(np.uint64)
        with dsss.tuned(sort_split_min=split_min):
            order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), p, part_begin=pb, small_sort_max=small)
        ro, rl = orc.local_sort(orc.Strings.from_host(hs), pb)
        assert np.array_equal(u64(order, n), ro)
        assert np.array_equal(u64(lcp, n), rl)


@pytest.mark.parametrize("graph", [0, 1 << 22])
def test_sort_split_pd(dsss, orc, ctx, graph):
    """The full path with splitter passes, host-driven and as one graph."""
    hs = dsss.gen_dn(200000, 60, 30, seed=41)
    with dsss.tuned(sort_split_min=4096, sort_graph_max_n=graph):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 4)
    check_pd(dsss, orc, hs, out, 4)


@pytest.mark.parametrize("bits,seg_bits", [(1, 1), (1, 0), (2, 1), (3, 1), (0, 0)])
@pytest.mark.parametrize("small", [0, 64])
@pytest.mark.parametrize("name,strs", CASES + _split_inputs(), ids=IDS + [c[0] for c in _split_inputs()])
def test_sort_bits(dsss, orc, ctx, name, strs, small, bits, seg_bits):
    """MSD passes that split plain keys on their eight most significant
    differing bits (sort_bits 1 for the passes over the arena, sort_seg_bits
    1 inside the segment sorter; several key bytes per pass over letters and
    DNA, strings that end inside a digit, bytes with a constant nonzero part)
    or on one key byte: the oracle's order and LCPs, in one segment and in
    three."""
    hs = host_of(dsss, strs)
    n = hs.n
    for p in (1, 3):
        if n < p:
            continue
        pb = np.linspace(0, n, p + 1).astype(np.uint64)
        with dsss.tuned(sort_bits=bits, sort_seg_bits=seg_bits):
            order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), p, part_begin=pb, small_sort_max=small)
        ro, rl = orc.local_sort(orc.Strings.from_host(hs), pb)
        assert np.array_equal(u64(order, n), ro)
        assert np.array_equal(u64(lcp, n), rl)


@pytest.mark.parametrize("seg_bits", [0, 1])
@pytest.mark.parametrize("graph", [0, 1 << 22])
@pytest.mark.parametrize("gen", ["dn", "suffix"])
def test_sort_bits_pd(dsss, orc, ctx, graph, gen, seg_bits):
    """The full path with bit-digit passes (D/N strings over letters and DNA
    suffixes), host-driven and as one graph, against the oracle."""
    hs = dsss.gen_dn(200000, 60, 30, seed=43) if gen == "dn" else dsss.gen_suffix_strings(120000, 256, seed=9)
    with dsss.tuned(sort_bits=1, sort_seg_bits=seg_bits, sort_graph_max_n=graph, sort_small_max=256):
        out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 4)
    check_pd(dsss, orc, hs, out, 4)
