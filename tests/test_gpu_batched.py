"""Batched form (dsss_pd_sort_batched): several independent string sets of
uneven sizes in one arena and one pipeline.  Every set's slice of the batched
result must equal the plain single-set result bit for bit, and the oracle's."""
import numpy as np
import pytest

from test_gpu_parity import check_pd, host_of, u64
from inputs import random_strings, with_duplicates

pytestmark = pytest.mark.gpu


def make_sets(dsss):
    return [
        dsss.gen_dn(40000, 100, 50, seed=21),
        dsss.gen_suffix_strings(30000, 256, seed=22),
        host_of(dsss, []),                                 # empty set
        dsss.gen_request(7000, seed=23),
        host_of(dsss, [b"a", b"b"]),                       # fewer strings than PEs
        dsss.gen_dn(40000, 100, 50, seed=21),              # same strings as set 0
        host_of(dsss, with_duplicates(random_strings(3000, 0, 40, b"ABC", seed=24), 0.3, seed=24)),
        dsss.gen_dn(12000, 60, 30, seed=25, long_len=300, long_k=200, frac_long=0.2),
    ]


def set_slice(out, sb, s, p):
    """Set s's part of a batched result, with arena ids made set-local."""
    b, e = int(sb[s]), int(sb[s + 1])
    n = e - b
    r = {}
    for k in ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp"):
        if out.get(k) is not None:
            v = u64(out[k], int(sb[-1]))[b:e]
            r[k] = v - b if k == "local_order" else v
    r["intervals"] = np.asarray(out["intervals"])[s * p * p:(s + 1) * p * p]
    r["recv_counts"] = np.asarray(out["recv_counts"])[s * p:(s + 1) * p]
    pb = np.asarray(out["part_begin"])[s * p:(s + 1) * p + 1] - np.uint64(b)
    r["part_begin"] = pb
    return r, n


def alone(dsss, ctx, hs, p, pb, sampler):
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), p, part_begin=pb, sampler=sampler)
    n = hs.n
    r = {k: u64(out[k], n)[:n] for k in ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp")}
    r["intervals"] = np.asarray(out["intervals"])
    r["recv_counts"] = np.asarray(out["recv_counts"])
    return r


@pytest.mark.parametrize("sampler", [0, 2])
@pytest.mark.parametrize("p", [1, 3, 8])
def test_batched_equals_alone(dsss, orc, ctx, p, sampler):
    sets = make_sets(dsss)
    hs, sb = dsss.concat_sets(sets)
    pb = dsss.batched_parts(sb, p)
    out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), len(sets), p, pb, sampler=sampler)
    for s, h in enumerate(sets):
        got, n = set_slice(out, sb, s, p)
        assert n == h.n
        if n == 0:
            assert not got["recv_counts"].any()
            continue
        ref = alone(dsss, ctx, h, p, got["part_begin"], sampler)
        assert np.array_equal(got["local_order"], ref["local_order"]), s
        assert np.array_equal(got["recv_counts"], ref["recv_counts"] if p > 1 else np.zeros(p, np.uint64)), s
        if p == 1:
            continue
        for k in ("dp", "perm_index", "perm_pe", "merged_lcp"):
            assert np.array_equal(got[k], ref[k]), (s, k)
        assert np.array_equal(got["intervals"], ref["intervals"]), s


@pytest.mark.parametrize("p", [4])
def test_batched_against_oracle(dsss, orc, ctx, p):
    sets = make_sets(dsss)
    hs, sb = dsss.concat_sets(sets)
    pb = dsss.batched_parts(sb, p)
    out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), len(sets), p, pb)
    for s, h in enumerate(sets):
        got, n = set_slice(out, sb, s, p)
        if n < p:
            continue
        check_pd(dsss, orc, h, got, p)


def test_batched_duplicate_sets_keep_their_dp(dsss, ctx):
    """Equal prefixes in different sets are not duplicates: a set batched with
    copies of itself gets the distinguishing prefixes it gets alone."""
    h = dsss.gen_dn(20000, 100, 50, seed=31)
    hs, sb = dsss.concat_sets([h, h, h])
    pb = dsss.batched_parts(sb, 4)
    out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), 3, 4, pb)
    ref = alone(dsss, ctx, h, 4, dsss.equal_parts(h.n, 4), 0)
    for s in range(3):
        got, _ = set_slice(out, sb, s, 4)
        assert np.array_equal(got["dp"], ref["dp"])
    assert set(ref["dp"].tolist()) == {72}


def test_batched_many_small_sets(dsss, orc, ctx):
    """256 sets of 0..500 random strings, p = 4 (1024 PEs in one call)."""
    rng = np.random.default_rng(41)
    sets = [host_of(dsss, random_strings(int(rng.integers(0, 500)), 0, 30, b"ABCD", seed=1000 + k))
            for k in range(256)]
    hs, sb = dsss.concat_sets(sets)
    pb = dsss.batched_parts(sb, 4)
    out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), len(sets), 4, pb)
    for s in range(0, 256, 17):
        got, n = set_slice(out, sb, s, 4)
        if n < 4:
            continue
        check_pd(dsss, orc, sets[s], got, 4)


def test_batched_host_matches_device(dsss, ctx):
    sets = make_sets(dsss)
    hs, sb = dsss.concat_sets(sets)
    pb = dsss.batched_parts(sb, 5)
    dev = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), len(sets), 5, pb)
    host = dsss.pd_sort_batched_host(ctx, hs, len(sets), 5, pb)
    n = hs.n
    for k in ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp"):
        assert np.array_equal(u64(dev[k], n), u64(host[k], n)), k
    assert np.array_equal(dev["intervals"], host["intervals"])
    assert np.array_equal(dev["recv_counts"], host["recv_counts"])


def test_batched_errors(dsss, ctx):
    h = dsss.gen_dn(1000, 20, 10, seed=1)
    hs, sb = dsss.concat_sets([h, h])
    ds = dsss.DeviceStrings(hs)
    with pytest.raises(dsss.DsssError) as e:  # too many PEs for one call
        dsss.pd_sort_batched(ctx, ds, 2, 600, dsss.batched_parts(sb, 600))
    assert e.value.code == -95
    with pytest.raises(dsss.DsssError) as e:  # bounds not covering the arena
        dsss.pd_sort_batched(ctx, ds, 2, 2, np.array([0, 10, 20, 30, 40], np.uint64))
    assert e.value.code == -22
