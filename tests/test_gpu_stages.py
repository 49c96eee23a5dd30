"""The stage entry points that mirror the reference's seams one by one
(BloomFilter::filter rounds, the PD exchange, the LCP merge), checked against
the oracle and the golden fixtures made from the reference, and chained in the
reference's own order (local sort -> DP -> partition -> exchange -> merge)."""
import json
import os

import numpy as np
import pytest
import torch

from inputs import cases, random_strings, with_duplicates

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def t32(a):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.uint32).view(np.int32)).cuda()


def u64(t):
    return t.cpu().numpy().view(np.uint32).astype(np.uint64)


CASES = [c for c in cases() if len(c[1]) >= 8]


@pytest.mark.parametrize("p", [1, 4])
@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_dp_round_by_round(dsss, orc, ctx, name, strs, p):
    hs = dsss.from_bytes_list(strs)
    n = hs.n
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(n, p)
    ro, rl = orc.local_sort(s, pb)
    rdp, rcounts = orc.dp_rounds(s, pb, ro, rl)
    ds = dsss.DeviceStrings(hs)
    order, lcp = t32(ro), t32(rl)
    results = torch.zeros(n, dtype=torch.int32, device="cuda")
    cand, depth, i, counts = None, 8, 16, []
    while True:
        cand, m = dsss.dp_round(ctx, ds, order, lcp, cand, depth, results)
        counts.append(m)
        if m == 0:
            break
        depth = 8 + i
        i *= 2
    assert counts == rcounts.tolist()
    assert np.array_equal(u64(results), rdp)


def staged(dsss, orc, hs, p):
    n = hs.n
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(n, p)
    ro, rl = orc.local_sort(s, pb)
    rdp, _ = orc.dp_rounds(s, pb, ro, rl)
    riv = orc.partition(s, pb, ro, rdp)
    return s, pb, ro, rl, rdp, riv


@pytest.mark.parametrize("p", [1, 2, 5, 8])
def test_bucket_scatter_matches_oracle(dsss, orc, ctx, p):
    strs = with_duplicates(random_strings(3000, 0, 30, b"ABCD", 100 + p), 0.2, 101)
    hs = dsss.from_bytes_list(strs)
    s, pb, ro, rl, rdp, riv = staged(dsss, orc, hs, p)
    ds = dsss.DeviceStrings(hs)
    g = dsss.bucket_scatter(ctx, ds, p, t32(ro), t32(rl), t32(rdp), riv)
    ex = orc.exchange(s, pb, ro, rl, rdp, riv)
    assert g["char_total"] == ex["chars"].size
    assert np.array_equal(g["chars"][:g["char_total"]].cpu().numpy(), ex["chars"])
    assert np.array_equal(g["char_begin"], ex["char_begin"])
    assert np.array_equal(u64(g["lcp"]), ex["lcp"])
    assert np.array_equal(u64(g["index"]), ex["index"])
    assert np.array_equal(u64(g["pe"]), ex["pe"])
    assert np.array_equal(g["counts"], ex["counts"])
    assert np.array_equal(g["offsets"], ex["offsets"])


def test_bucket_scatter_kat(dsss, ctx):
    """src/tests/alltoallStrings_tests.cpp:129-163 through the device scatter."""
    with open(os.path.join(GOLDEN, "pd_exchange_kat.json")) as f:
        kat = json.load(f)
    for case in kat:
        p = case["p"]
        strs, lcps, dps, sends = [], [], [], []
        for pe in case["pes"]:
            strs += [bytes.fromhex(x) for x in pe["strings"]]
            lcps += pe["lcp"]
            dps += pe["dp"]
            sends.append(pe["send"])
        hs = dsss.from_bytes_list(strs)
        n = hs.n
        ds = dsss.DeviceStrings(hs)
        g = dsss.bucket_scatter(ctx, ds, p, t32(np.arange(n)), t32(lcps), t32(dps), np.array(sends))
        m = len(case["expected_lcp"])
        chars = g["chars"].cpu().numpy()
        for r in range(p):
            cb, ce = int(g["char_begin"][r]), int(g["char_begin"][r + 1])
            assert chars[cb:ce].tobytes().hex() == case["expected_raw"], (p, r)
            assert u64(g["lcp"])[r * m:(r + 1) * m].tolist() == case["expected_lcp"], (p, r)


def string_runs_equal(strs_got, strs_ref, labels_got, labels_ref):
    """Same strings in the same order; labels may permute only within runs of equal strings."""
    assert strs_got == strs_ref
    n = len(strs_ref)
    k = 0
    while k < n:
        e = k + 1
        while e < n and strs_ref[e] == strs_ref[k]:
            e += 1
        assert sorted(labels_got[k:e]) == sorted(labels_ref[k:e])
        k = e


@pytest.mark.parametrize("by_sort", [1, 0, 2])
def test_lcp_merge_golden(dsss, ctx, by_sort):
    """merge_ref.json: the reference's LcpStringLoserTree_ on receive containers
    (runs merged by one segmented sort, by merge-path rounds, or all at once
    by co-ranked tiles)."""
    with open(os.path.join(GOLDEN, "merge_ref.json")) as f:
        gold = json.load(f)
    with dsss.tuned(merge_by_sort=by_sort):
        _merge_golden(dsss, ctx, gold)


def _merge_golden(dsss, ctx, gold):
    for name, v in gold.items():
        for pe in v["pes"]:
            raw = bytes.fromhex(pe["chars"])
            n = len(pe["lcp"])
            chars = torch.from_numpy(np.frombuffer(raw + b"\0" * 64, np.uint8).copy()).cuda()
            out = dsss.lcp_merge(ctx, chars, len(raw), t32(pe["lcp"]), np.array([pe["counts"]]),
                                 np.array([pe["offsets"]]))
            # strings of the container, decompressed on the host for the comparison
            starts, full, prev = [], [], b""
            pos = 0
            for _ in range(n):
                e = raw.index(b"\0", pos)
                starts.append(pos)
                pos = e + 1
            k = 0
            run_first = set()
            for c in pe["counts"]:
                if c:
                    run_first.add(k)
                k += c
            for o in range(n):
                comp = raw[starts[o]:raw.index(b"\0", starts[o])]
                l = 0 if o in run_first else pe["lcp"][o]
                cur = prev[:l] + comp
                full.append(cur)
                prev = cur
            order = u64(out["order"])
            got_s = [full[int(o)] for o in order]
            idx, src = u64(out["perm_index"]), u64(out["perm_pe"])
            ref_labels = list(zip(pe["index"], pe["pe"], pe["old_lcp"]))
            got_labels = list(zip(idx.tolist(), src.tolist(), u64(out["old_lcp"]).tolist()))
            ref_s = sorted(full)
            string_runs_equal(got_s, ref_s, got_labels, ref_labels)
            assert u64(out["merged_lcp"]).tolist() == pe["merged_lcp"], name


@pytest.mark.parametrize("by_sort", [1, 0, 2])
@pytest.mark.parametrize("p", [2, 3, 4, 8, 16])
def test_staged_pipeline_matches_oracle(dsss, orc, ctx, p, by_sort):
    """The reference's stage order on the GPU: local sort, DP rounds, partition,
    bucket scatter, LCP merge of every PE's container."""
    strs = with_duplicates(random_strings(6000, 0, 40, b"ABC", 200 + p), 0.15, 201)
    hs = dsss.from_bytes_list(strs)
    n = hs.n
    ds = dsss.DeviceStrings(hs)
    pb = dsss.equal_parts(n, p)
    order, lcp = dsss.local_sort_lcp(ctx, ds, p)
    dp, _ = dsss.dp_prefixes(ctx, ds, order, lcp, p)
    iv = dsss.partition(ctx, ds, order, dp, p)
    g = dsss.bucket_scatter(ctx, ds, p, order, lcp, dp, iv)
    with dsss.tuned(merge_by_sort=by_sort):
        out = dsss.lcp_merge(ctx, g["chars"], g["char_total"], g["lcp"], g["counts"], g["offsets"],
                             char_start=g["char_start"])
    r = orc.pd_sort(orc.Strings.from_host(hs), pb)
    assert np.array_equal(iv, r["intervals"])
    local = u64(order)
    assert np.array_equal(local, r["order"])

    def sof(i, q):
        return strs[int(local[int(pb[int(q)]) + int(i)])]

    gi, gp = u64(out["perm_index"]), u64(out["perm_pe"])
    got_s = [sof(i, q) for i, q in zip(gi, gp)]
    ref_s = [sof(i, q) for i, q in zip(r["perm_index"], r["perm_pe"])]
    string_runs_equal(got_s, ref_s, list(zip(gp.tolist(), gi.tolist())),
                      list(zip(r["perm_pe"].tolist(), r["perm_index"].tolist())))
    # merged LCP restarts at 0 for every receiving PE
    assert np.array_equal(u64(out["merged_lcp"]), r["merged_lcp"])


def test_lcp_merge_modes_identical(dsss, ctx):
    """Sort-based and merge-path merging give the same order, LCPs and labels
    (ties in run order) on containers with many byte-identical strings."""
    hs = dsss.gen_suffix_strings(200000, 256, seed=12)
    ds = dsss.DeviceStrings(hs)
    p = 8
    order, lcp = dsss.local_sort_lcp(ctx, ds, p)
    dp, _ = dsss.dp_prefixes(ctx, ds, order, lcp, p)
    iv = dsss.partition(ctx, ds, order, dp, p)
    g = dsss.bucket_scatter(ctx, ds, p, order, lcp, dp, iv)
    outs = []
    for m in (1, 0, 2):
        with dsss.tuned(merge_by_sort=m):
            outs.append(dsss.lcp_merge(ctx, g["chars"], g["char_total"], g["lcp"], g["counts"], g["offsets"],
                                       char_start=g["char_start"]))
    for k in ("order", "merged_lcp", "old_lcp", "perm_index", "perm_pe"):
        for o in outs[1:]:
            assert np.array_equal(u64(outs[0][k]), u64(o[k])), k


@pytest.mark.parametrize("which", ["dn", "suffix", "equal", "skewed"])
def test_lcp_merge_kway_many_runs(dsss, ctx, which):
    """The K-way merge by co-ranked tiles on receive containers of 16 to 64
    runs each, with tiles that cut runs of byte-identical strings (suffixes,
    all-equal strings) and runs of very different lengths: the same order,
    LCPs and labels as the merge by one sort."""
    if which == "dn":
        hs, p = dsss.gen_dn(1500000, 60, 30, seed=14), 64
    elif which == "suffix":
        hs, p = dsss.gen_suffix_strings(400000, 256, seed=15), 16
    elif which == "equal":
        hs, p = dsss.from_bytes_list([b"SAME" * 5] * 300000), 32
    else:
        rng = np.random.default_rng(16)
        hs, p = dsss.from_bytes_list([bytes(rng.integers(65, 70, int(k)).astype(np.uint8))
                                      for k in rng.integers(0, 12, 200000)]), 24
    ds = dsss.DeviceStrings(hs)
    n = hs.n
    # uneven PEs (an empty one among them when two cuts meet)
    cuts = np.sort(np.random.default_rng(17).integers(0, n, p - 1))
    pb = np.concatenate([[0], cuts, [n]]).astype(np.uint64)
    order, lcp = dsss.local_sort_lcp(ctx, ds, p, part_begin=pb)
    dp, _ = dsss.dp_prefixes(ctx, ds, order, lcp, p, part_begin=pb)
    iv = dsss.partition(ctx, ds, order, dp, p, part_begin=pb)
    g = dsss.bucket_scatter(ctx, ds, p, order, lcp, dp, iv, part_begin=pb)
    outs = []
    for m in (1, 2):
        with dsss.tuned(merge_by_sort=m):
            outs.append(dsss.lcp_merge(ctx, g["chars"], g["char_total"], g["lcp"], g["counts"], g["offsets"],
                                       char_start=g["char_start"]))
    for k in ("order", "merged_lcp", "old_lcp", "perm_index", "perm_pe"):
        assert np.array_equal(u64(outs[0][k]), u64(outs[1][k])), k


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_lcp_merge_extend_lanes(dsss, ctx, lanes):
    """Prefix decompression with 4..32 threads per chunk of strings gives the golden
    merge results, and the same order as the automatic choice on long shared
    prefixes (suffixes of a 256-byte-periodic text)."""
    with open(os.path.join(GOLDEN, "merge_ref.json")) as f:
        gold = json.load(f)
    with dsss.tuned(merge_extend_lanes=lanes):
        _merge_golden(dsss, ctx, gold)
    hs = dsss.gen_suffix_strings(50000, 256, seed=13)
    ds = dsss.DeviceStrings(hs)
    p = 4
    order, lcp = dsss.local_sort_lcp(ctx, ds, p)
    dp, _ = dsss.dp_prefixes(ctx, ds, order, lcp, p)
    iv = dsss.partition(ctx, ds, order, dp, p)
    g = dsss.bucket_scatter(ctx, ds, p, order, lcp, dp, iv)
    outs = []
    for k in (0, lanes):
        with dsss.tuned(merge_extend_lanes=k):
            outs.append(dsss.lcp_merge(ctx, g["chars"], g["char_total"], g["lcp"], g["counts"], g["offsets"],
                                       char_start=g["char_start"]))
    for k in ("order", "merged_lcp", "old_lcp", "perm_index", "perm_pe"):
        assert np.array_equal(u64(outs[0][k]), u64(outs[1][k])), k
