"""Exact parity with the oracle at the benchmark sizes: the GPU's full
prefix-doubling path against the oracle's restatement on the same inputs,
every output compared (local orders, distinguishing-prefix lengths, interval
tables, receive counts, merged LCPs and the (index, PE) permutation; labels of
byte-identical strings compared as sets within their run):

  - 32e6 strings x 200 B, D/N 0.25, p = 64 (the benchmark's main workload);
  - 1e8 strings x 100 B, D/N 0.5, p = 64;
  - the skewed set: 20e6 strings, 20 % x 500 B (k = 400), p = 64;
  - one full suffix set: all 2^26 suffixes (x 256 B) of a 64 MiB text, p = 64;
  - every set of the batched form's 16 x 4 MiB suffix batch, p = 64 each.

The oracle is single-threaded (about 1e6 strings/s); it runs in a worker
thread while the GPU computes, and independent oracle runs share a thread
pool."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from test_gpu_parity import u64

pytestmark = pytest.mark.gpu

P = 64


def check_big(hs, out, r, p):
    """check_pd for large inputs: vectorised comparison, ties between
    byte-identical strings compared per run as label multisets."""
    n = hs.n
    assert np.array_equal(u64(out["local_order"], n), r["order"])
    assert np.array_equal(u64(out["dp"], n), r["dp"])
    assert np.array_equal(np.asarray(out["intervals"]).reshape(p, p), r["intervals"])
    assert np.array_equal(np.asarray(out["recv_counts"]), r["recv_counts"])
    assert np.array_equal(u64(out["merged_lcp"], n), r["merged_lcp"])
    gi, gp = u64(out["perm_index"], n), u64(out["perm_pe"], n)
    ri, rp = r["perm_index"], r["perm_pe"]
    if np.array_equal(gi, ri) and np.array_equal(gp, rp):
        return
    # the merged strings' lengths (reference labels)
    pb = np.asarray(out["part_begin"], np.uint64)
    sid = r["order"][(pb[rp.astype(np.int64)] + ri).astype(np.int64)]
    L = hs.lengths[sid.astype(np.int64)].astype(np.uint64)
    tie = np.zeros(n, bool)
    tie[1:] = (r["merged_lcp"][1:] == L[1:]) & (L[1:] == L[:-1])
    starts = np.concatenate([[0], np.cumsum(r["recv_counts"].astype(np.int64))[:-1]])
    tie[starts[starts < n]] = False
    bad = (gi != ri) | (gp != rp)
    assert not (bad & ~tie & ~np.roll(tie, -1)).any(), "a label differs outside a run of byte-identical strings"
    run = np.cumsum(~tie)
    lab_g = gp.astype(np.uint64) << np.uint64(40) | gi
    lab_r = rp.astype(np.uint64) << np.uint64(40) | ri
    og = np.lexsort((lab_g, run))
    orr = np.lexsort((lab_r, run))
    assert np.array_equal(lab_g[og], lab_r[orr])


@pytest.fixture(scope="module")
def pool():
    ex = cf.ThreadPoolExecutor(max_workers=max(2, min(16, (os.cpu_count() or 2) - 1)))
    yield ex
    ex.shutdown()


def oracle_async(pool, orc, hs, pb):
    s = orc.Strings.from_host(hs)
    return pool.submit(orc.pd_sort, s, np.asarray(pb, np.uint64))


@pytest.mark.parametrize("n,length,k,gk", [
    (32_000_000, 200, 50, {}),
    (100_000_000, 100, 50, {}),
    (20_000_000, 100, 20, dict(long_len=500, long_k=400, frac_long=0.2)),
], ids=["dn32m", "dn100m", "skew20m"])
def test_full_size_against_oracle(dsss, orc, ctx, pool, n, length, k, gk):
    hs = dsss.gen_dn(n, length, k, seed=1, **gk)
    pb = dsss.equal_parts(n, P)
    fut = oracle_async(pool, orc, hs, pb)
    ds = dsss.DeviceStrings(hs)
    out = dsss.pd_sort(ctx, ds, P)
    out = {kk: (v.cpu() if hasattr(v, "cpu") else v) for kk, v in out.items()}
    del ds
    check_big(hs, out, fut.result(), P)


def test_full_suffix_set_against_oracle(dsss, orc, ctx, pool):
    hs = dsss.gen_suffix_strings(64 << 20, 256, seed=1)
    pb = dsss.equal_parts(hs.n, P)
    fut = oracle_async(pool, orc, hs, pb)
    out = dsss.pd_sort(ctx, dsss.DeviceStrings(hs), P)
    out = {kk: (v.cpu() if hasattr(v, "cpu") else v) for kk, v in out.items()}
    check_big(hs, out, fut.result(), P)


def test_batched_suffix_sets_against_oracle(dsss, orc, ctx, pool):
    """The batched benchmark's 16 instances (4 MiB texts, seeds 100..115): every
    set's slice of one batched call equals the oracle's run on that set."""
    from test_gpu_batched import set_slice
    sets = [dsss.gen_suffix_strings(4 << 20, 256, seed=100 + s) for s in range(16)]
    hs, sb = dsss.concat_sets(sets)
    pbs = dsss.batched_parts(sb, P)
    futs = []
    for s, h in enumerate(sets):
        futs.append(oracle_async(pool, orc, h, dsss.equal_parts(h.n, P)))
    out = dsss.pd_sort_batched(ctx, dsss.DeviceStrings(hs), len(sets), P, pbs)
    out = {kk: (v.cpu() if hasattr(v, "cpu") else v) for kk, v in out.items()}
    for s, h in enumerate(sets):
        got, n = set_slice(out, sb, s, P)
        assert n == h.n
        assert np.array_equal(got["part_begin"], dsss.equal_parts(h.n, P).astype(np.uint64))
        check_big(h, dict(got, local_order=got["local_order"]), futs[s].result(), P)
