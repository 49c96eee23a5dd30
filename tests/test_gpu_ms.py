"""dsss_ms_sort (the merge-sort path, DistributedMergeSort::sort) against the
oracle's restatement: average LCP, interval table, strings per receiving PE,
local orders, and every output string (bytes, length, offset) with its LCP.
Byte-identical strings are indistinguishable in this output, so `source` is
compared through the bytes it names."""
import numpy as np
import pytest

from inputs import cases
from test_gpu_parity import host_of, u64
from test_ms_oracle import truncation_case

pytestmark = pytest.mark.gpu

CASES = [c for c in cases() if len(c[1]) >= 8]
IDS = [c[0] for c in CASES]


def check_ms(dsss, orc, hs, out, pb):
    n = hs.n
    s = orc.Strings.from_host(hs)
    r = orc.ms_sort(s, pb)
    p = len(pb) - 1
    assert out["avg_lcp"] == r["avg_lcp"]
    assert np.array_equal(np.asarray(out["intervals"]).reshape(p, p), r["intervals"])
    assert np.array_equal(np.asarray(out["recv_counts"]), r["recv_counts"])
    assert np.array_equal(u64(out["local_order"], n), r["order"])
    if n == 0:
        return
    lens = u64(out["lengths"], n)
    offs = out["offsets"][:n].cpu().numpy().astype(np.int64)
    chars = out["chars"].cpu().numpy()
    src = u64(out["source"], n)
    want = [s.get(int(i)) for i in r["source"]]
    got = [chars[o:o + int(l)].tobytes() for o, l in zip(offs, lens)]
    assert got == want
    assert all(chars[o + int(l)] == 0 for o, l in zip(offs, lens))
    assert [s.get(int(i)) for i in src] == want
    assert np.array_equal(u64(out["lcp"], n), r["out_lcp"])
    # back to back: each string starts where the previous one's NUL ends
    assert offs[0] == 0 and np.array_equal(offs[1:], offs[:-1] + lens[:-1].astype(np.int64) + 1)


@pytest.mark.parametrize("p", [1, 3, 8])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_ms_sort_matches_oracle(dsss, orc, ctx, name, strs, p):
    hs = host_of(dsss, strs)
    if hs.n < p:
        pytest.skip("fewer strings than PEs")
    pb = np.linspace(0, hs.n, p + 1).astype(np.uint64)
    out = dsss.ms_sort(ctx, dsss.DeviceStrings(hs), p, part_begin=pb)
    check_ms(dsss, orc, hs, out, pb)


@pytest.mark.parametrize("p", [4, 16])
def test_ms_sort_dn_and_suffixes(dsss, orc, ctx, p):
    for hs in (dsss.gen_dn(60000, 100, 50, seed=p), dsss.gen_suffix_strings(60000, 256, seed=p)):
        pb = dsss.equal_parts(hs.n, p).astype(np.uint64)
        out = dsss.ms_sort(ctx, dsss.DeviceStrings(hs), p, part_begin=pb)
        check_ms(dsss, orc, hs, out, pb)


def test_ms_sort_truncated_splitter(dsss, orc, ctx):
    """Samples cut at 200 (avg + 5) bytes move a string across the splitter
    (the case the oracle test derives by hand: PE 0 keeps 999 strings)."""
    strs, pb = truncation_case()
    hs = host_of(dsss, strs)
    out = dsss.ms_sort(ctx, dsss.DeviceStrings(hs), 2, part_begin=pb)
    assert np.asarray(out["intervals"]).reshape(2, 2)[0].tolist() == [999, 2001]
    check_ms(dsss, orc, hs, out, pb)


@pytest.mark.parametrize("strs,pb", [
    ([], [0, 0, 0]),
    ([b"solo"], [0, 1]),
    ([b"solo"], [0, 0, 1, 1]),                       # empty PEs around one string
    ([b"", b"", b"a", b""], [0, 2, 4]),              # empty strings
    ([b"b", b"a", b"c"], [0, 1, 1, 2, 2, 3]),        # p = 5 > n with empty PEs
])
def test_ms_sort_edges(dsss, orc, ctx, strs, pb):
    hs = host_of(dsss, strs)
    pb = np.asarray(pb, np.uint64)
    out = dsss.ms_sort(ctx, dsss.DeviceStrings(hs), len(pb) - 1, part_begin=pb)
    check_ms(dsss, orc, hs, out, pb)
