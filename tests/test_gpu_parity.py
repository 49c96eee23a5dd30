"""Parity of the CUDA path (through the C ABI) with the oracle, stage by stage
and end to end.  Integer work: every comparison is exact.  The only freedom
is the order among byte-identical strings in the merged output, which the
reference's loser tree decides by tournament history; there the (PE, index)
labels are compared as sets per run of identical strings."""
import numpy as np
import pytest

from inputs import cases, long_prefix, random_strings, with_duplicates

pytestmark = pytest.mark.gpu


def host_of(dsss, strs):
    return dsss.from_bytes_list(strs)


def u64(t, n=None):
    a = t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)
    a = a.view(np.uint32) if a.dtype == np.int32 else a
    a = a.astype(np.uint64)
    return a if n is None else a[:n]


CASES = cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("depth", [0, 1, 7, 8, 24, 31, 32, 33, 40, 64, 72, 136, 264, 600])
def test_prefix_hash(dsss, orc, depth):
    import torch
    strs = random_strings(3000, 0, 620, bytes(range(1, 256)), 50 + depth)
    hs = host_of(dsss, strs)
    ds = dsss.DeviceStrings(hs)
    ids = torch.arange(hs.n, dtype=torch.int32, device="cuda")
    h = dsss.prefix_hash(ds, ids, depth).cpu().numpy().view(np.uint64)
    M = (1 << 64) - 1
    for i, s in enumerate(strs):
        assert int(h[i]) == orc.xxh64(s[:depth]) % M, (i, len(s))


@pytest.mark.parametrize("small_max", [0, 2, 32, 300])
@pytest.mark.parametrize("p", [1, 3])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_local_sort(dsss, orc, ctx, name, strs, p, small_max):
    hs = host_of(dsss, strs)
    n = hs.n
    if n < p:
        pytest.skip("fewer strings than PEs")
    ds = dsss.DeviceStrings(hs)
    order, lcp = dsss.local_sort_lcp(ctx, ds, p, small_sort_max=small_max)
    s = orc.Strings.from_host(hs)
    ro, rl = orc.local_sort(s, dsss.equal_parts(n, p))
    assert np.array_equal(u64(order, n), ro)
    assert np.array_equal(u64(lcp, n), rl)


@pytest.mark.parametrize("p", [1, 4])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_dp_prefixes(dsss, orc, ctx, name, strs, p):
    import torch
    hs = host_of(dsss, strs)
    n = hs.n
    if n < p:
        pytest.skip("fewer strings than PEs")
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(n, p)
    ro, rl = orc.local_sort(s, pb)
    rdp, rcounts = orc.dp_rounds(s, pb, ro, rl)
    ds = dsss.DeviceStrings(hs)
    order = torch.from_numpy(ro.astype(np.int32)).cuda()
    lcp = torch.from_numpy(rl.astype(np.int32)).cuda()
    dp, counts = dsss.dp_prefixes(ctx, ds, order, lcp, p)
    assert np.array_equal(u64(dp, n), rdp)
    assert counts.tolist() == rcounts.tolist()


@pytest.mark.parametrize("sampler", [0, 2])
@pytest.mark.parametrize("p", [2, 5, 16])
def test_partition(dsss, orc, ctx, p, sampler):
    import torch
    strs = with_duplicates(random_strings(4000, 0, 24, b"ABCD", 60 + p), 0.2, 61)
    hs = host_of(dsss, strs)
    n = hs.n
    s = orc.Strings.from_host(hs)
    pb = dsss.equal_parts(n, p)
    ro, rl = orc.local_sort(s, pb)
    rdp, _ = orc.dp_rounds(s, pb, ro, rl)
    riv = orc.partition(s, pb, ro, rdp, indexed=sampler == 2)
    ds = dsss.DeviceStrings(hs)
    iv = dsss.partition(ctx, ds, torch.from_numpy(ro.astype(np.int32)).cuda(),
                        torch.from_numpy(rdp.astype(np.int32)).cuda(), p, sampler=sampler)
    assert np.array_equal(iv, riv)


@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_adjacent_lcp(dsss, orc, ctx, name, strs):
    import torch
    hs = host_of(dsss, strs)
    n = hs.n
    s = orc.Strings.from_host(hs)
    ro, rl = orc.local_sort(s, np.array([0, n], np.uint64))
    ds = dsss.DeviceStrings(hs)
    lcp = dsss.adjacent_lcp(ctx, ds, torch.from_numpy(ro.astype(np.int32)).cuda())
    assert np.array_equal(u64(lcp, n), rl)


def check_pd(dsss, orc, hs, out, p, indexed=False):
    """Compares a dsss_pd_sort result with the oracle's full path."""
    n = hs.n
    s = orc.Strings.from_host(hs)
    r = orc.pd_sort(s, out["part_begin"], indexed=indexed)
    assert np.array_equal(u64(out["local_order"], n), r["order"])
    if p == 1:
        assert list(out["recv_counts"]) == [0]
        return
    assert np.array_equal(u64(out["dp"], n), r["dp"])
    assert np.array_equal(np.asarray(out["intervals"]).reshape(p, p), r["intervals"])
    assert np.array_equal(np.asarray(out["recv_counts"]), r["recv_counts"])
    if out.get("merged_lcp") is not None:
        assert np.array_equal(u64(out["merged_lcp"], n), r["merged_lcp"])
    gi, gp = u64(out["perm_index"], n), u64(out["perm_pe"], n)
    if np.array_equal(gi, r["perm_index"]) and np.array_equal(gp, r["perm_pe"]):
        return
    # Only runs of byte-identical strings may differ in label order.
    pb = out["part_begin"]
    order = r["order"]

    def string_of(q, i):
        return s.get(int(order[int(pb[int(q)]) + int(i)]))

    ref_str = [string_of(q, i) for i, q in zip(r["perm_index"], r["perm_pe"])]
    got_str = [string_of(q, i) for i, q in zip(gi, gp)]
    assert got_str == ref_str
    k = 0
    while k < n:
        e = k + 1
        while e < n and ref_str[e] == ref_str[k]:
            e += 1
        assert sorted(zip(gp[k:e], gi[k:e])) == sorted(zip(r["perm_pe"][k:e], r["perm_index"][k:e]))
        k = e


@pytest.mark.parametrize("sampler", [0, 2])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_pd_sort_cases(dsss, orc, ctx, name, strs, p, sampler):
    hs = host_of(dsss, strs)
    if hs.n < p:
        pytest.skip("fewer strings than PEs")
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p, sampler=sampler)
    check_pd(dsss, orc, hs, out, p, indexed=sampler == 2)


@pytest.mark.parametrize("p", [2, 4, 16, 64])
def test_pd_sort_dn(dsss, orc, ctx, p):
    """Strings of the D/N rule of the 1e6 x 100 B configuration, smaller."""
    hs = dsss.gen_dn(200000, 100, 50, seed=p)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p)
    check_pd(dsss, orc, hs, out, p)


def test_pd_sort_c1_full(dsss, orc, ctx):
    """n = 1e6 strings of 100 bytes, D/N 0.5, p = 4 (the reference's plain configuration)."""
    hs = dsss.gen_dn(1000000, 100, 50, seed=1)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 4)
    check_pd(dsss, orc, hs, out, 4)
    assert set(u64(out["dp"], hs.n).tolist()) == {72}


def test_pd_sort_skewed(dsss, orc, ctx):
    """Skewed D/N: 20% of the strings 500 bytes (D/N 0.8), the rest 100 (D/N 0.2)."""
    hs = dsss.gen_dn(100000, 100, 20, seed=3, long_len=500, long_k=400, frac_long=0.2)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 8)
    check_pd(dsss, orc, hs, out, 8)


@pytest.mark.parametrize("p", [1, 4, 16])
def test_pd_sort_suffixes(dsss, orc, ctx, p):
    """All suffixes (truncated to 256 bytes) of a Markov text with copied blocks:
    long LCPs and many byte-identical strings."""
    hs = dsss.gen_suffix_strings(150000, 256, seed=5)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p)
    check_pd(dsss, orc, hs, out, p)


@pytest.mark.parametrize("which", ["suffix_1mib", "request_300k"])
def test_local_sort_long_chains(dsss, orc, ctx, which):
    """Inputs whose sort tree has long chains of large groups (repeats in a
    suffix set; strings sharing a random-length common head): the pivot
    passes of the sort, checked against the oracle's order and LCPs."""
    hs = dsss.gen_suffix_strings(1 << 20, 256, seed=100) if which == "suffix_1mib" else dsss.gen_request(300000, seed=3)
    n = hs.n
    order, lcp = dsss.local_sort_lcp(ctx, dsss.DeviceStrings(hs), 1)
    ro, rl = orc.local_sort(orc.Strings.from_host(hs), np.array([0, n], np.uint64))
    assert np.array_equal(u64(order, n), ro)
    assert np.array_equal(u64(lcp, n), rl)


def test_pd_sort_request(dsss, orc, ctx):
    hs = dsss.gen_request(50000, seed=9)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 8)
    check_pd(dsss, orc, hs, out, 8)


def test_pd_sort_host_matches_device(dsss, orc, ctx):
    hs = dsss.gen_dn(50000, 80, 40, seed=11)
    dev = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 5)
    host = dsss.pd_sort_host(ctx, hs, 5)
    n = hs.n
    for k in ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp"):
        assert np.array_equal(u64(dev[k], n), u64(host[k], n)), k
    assert np.array_equal(dev["intervals"], host["intervals"])
    check_pd(dsss, orc, hs, host, 5)


def test_pd_sort_uneven_parts(dsss, orc, ctx):
    """PEs of unequal (and empty) size, as byte-slice input distribution gives."""
    hs = dsss.gen_dn(30000, 50, 25, seed=13)
    pb = np.array([0, 0, 1000, 1000, 17000, 29999, 30000], np.uint64)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), 6, part_begin=pb)
    check_pd(dsss, orc, hs, out, 6)


def test_errors(dsss, ctx):
    hs = dsss.gen_dn(100, 20, 10, seed=1)
    ds = dsss.DeviceStrings(hs)
    with pytest.raises(dsss.DsssError) as e:
        dsss.pd_sort(ctx, ds, 2, part_begin=np.array([0, 10, 50], np.uint64))
    assert e.value.code == -22
    with pytest.raises(dsss.DsssError):
        dsss.pd_sort(ctx, ds, 0, part_begin=np.array([100], np.uint64))


def test_budget_enomem(dsss):
    small = dsss.Context(0, hbm_budget=1 << 16)
    hs = dsss.gen_dn(100000, 50, 25, seed=1)
    with pytest.raises(dsss.DsssError) as e:
        dsss.pd_sort(small, dsss.DeviceStrings(hs), 4)
    assert e.value.code == -12
    small.close()


@pytest.mark.parametrize("kind", ["distinct", "ties"])
def test_merged_sequences_direct_and_multisplit(dsss, orc, ctx, kind):
    """When every bucket follows the previous one along the global order, the
    merged sequences are written directly (one multisplit per call, the one by
    PE); equal strings that PEs cut on different sides of a splitter force the
    stable multisplit by bucket (two per call).  The oracle's full path either
    way."""
    rng = np.random.default_rng(21)
    if kind == "distinct":
        strs = [bytes(rng.integers(65, 91, size=12, dtype=np.uint8)) for _ in range(6000)]
    else:
        strs = [b"SAME" if rng.random() < 0.6 else bytes(rng.integers(65, 68, size=3, dtype=np.uint8))
                for _ in range(6000)]
    hs = host_of(dsss, strs)
    p = 8
    ctx.set_timing(True)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p)
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    assert kt["k_ms_scatter_pay"][0] == (1 if kind == "distinct" else 2)
    check_pd(dsss, orc, hs, out, p)
