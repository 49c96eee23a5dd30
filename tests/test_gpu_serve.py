"""Request server (dsss_server_*): continuous batching of sort requests.  Each
request's result must be the same alone (dsss_pd_sort_host) and in the mix,
bit for bit; admission must keep the reserved device memory within the budget."""
import numpy as np
import pytest

from test_gpu_parity import check_pd, u64

pytestmark = pytest.mark.gpu

KEYS = ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp")


def requests(dsss, count, seed, lo=1000, hi=200000):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)
    return [dsss.gen_request(int(n), seed=seed * 1000 + k) for k, n in enumerate(ns)]


def assert_same(a, b, n, p):
    assert np.array_equal(u64(a["local_order"], n), u64(b["local_order"], n))
    assert np.array_equal(np.asarray(a["recv_counts"]), np.asarray(b["recv_counts"]))
    if p == 1:
        return
    for k in KEYS[1:]:
        assert np.array_equal(u64(a[k], n), u64(b[k], n)), k
    assert np.array_equal(np.asarray(a["intervals"]), np.asarray(b["intervals"]))


@pytest.mark.parametrize("p", [1, 4, 16])
def test_server_same_alone_and_in_the_mix(dsss, ctx, p):
    reqs = requests(dsss, 24, seed=p)
    srv = dsss.Server(0, p=p, workers=2, max_sets=8)
    tickets = [srv.submit(h) for h in reqs]
    stats = [srv.wait(t) for t, _ in tickets]
    info = srv.info()
    srv.close()
    assert info["batched_requests"] == len(reqs)
    assert info["batches"] < len(reqs)           # requests were batched together
    assert max(s["batch_sets"] for s in stats) > 1
    for h, (t, out) in zip(reqs, tickets):
        alone = dsss.pd_sort_host(ctx, h, p)
        assert_same(out, alone, h.n, p)


def test_server_against_oracle(dsss, orc, ctx):
    reqs = requests(dsss, 6, seed=77, lo=500, hi=20000)
    srv = dsss.Server(0, p=4, workers=3, max_sets=4)
    tickets = [srv.submit(h) for h in reqs]
    for t, _ in tickets:
        srv.wait(t)
    srv.close()
    for h, (t, out) in zip(reqs, tickets):
        check_pd(dsss, orc, h, out, 4)


def test_server_budget_admission(dsss, ctx):
    reqs = requests(dsss, 12, seed=5, lo=20000, hi=100000)
    probe = dsss.Server(0, p=4)
    need = max(probe.footprint(h.n, h.char_bytes) for h in reqs)
    probe.close()
    budget = int(need * 1.5)                      # room for one request at a time, sometimes two
    srv = dsss.Server(0, p=4, workers=3, max_sets=8, hbm_budget=budget)
    tickets = [srv.submit(h) for h in reqs]
    for t, _ in tickets:
        srv.wait(t)
    info = srv.info()
    assert 0 < info["max_reserved_bytes"] <= budget
    assert info["reserved_bytes"] == 0
    for h, (t, out) in zip(reqs, tickets):
        assert_same(out, dsss.pd_sort_host(ctx, h, 4), h.n, 4)
    big = dsss.gen_request(400000, seed=9)
    t, _ = srv.submit(big)
    with pytest.raises(dsss.DsssError) as e:
        srv.wait(t)
    assert e.value.code == -12
    srv.close()


def test_server_uneven_parts_and_empty(dsss, ctx):
    srv = dsss.Server(0, p=3, workers=2)
    h1 = dsss.gen_request(5000, seed=3)
    pb = np.array([0, 0, 4000, 5000], np.uint64)
    h2 = dsss.from_bytes_list([])
    h3 = dsss.from_bytes_list([b"x"])
    t1, o1 = srv.submit(h1, part_begin=pb)
    t2, o2 = srv.submit(h2)
    t3, o3 = srv.submit(h3)
    for t in (t1, t2, t3):
        srv.wait(t)
    srv.close()
    assert_same(o1, dsss.pd_sort_host(ctx, h1, 3, part_begin=pb), h1.n, 3)
    assert not np.asarray(o2["recv_counts"]).any()
    assert_same(o3, dsss.pd_sort_host(ctx, h3, 3), 1, 3)


def test_server_wait_timeout_keeps_ticket(dsss):
    srv = dsss.Server(0, p=4, workers=1)
    h = dsss.gen_request(300000, seed=4)
    t, _ = srv.submit(h)
    try:
        srv.wait(t, timeout_ms=0)
    except dsss.DsssError as e:
        assert e.code == -110
        srv.wait(t)                               # still valid after a timeout
    with pytest.raises(dsss.DsssError):
        srv.wait(t)                               # released
    srv.close()
