"""dsss_hq_sort (hQuicksort: RQuick::sort as the reference's executable runs
it) against the oracle's restatement: strings per PE, every output string
(bytes, length, offset) in order, and the strings `source` names.
Byte-identical strings are indistinguishable in this output, so `source` is
compared through the bytes it names."""
import numpy as np
import pytest

from inputs import cases
from test_gpu_parity import host_of, u64

pytestmark = pytest.mark.gpu

CASES = [c for c in cases() if len(c[1]) >= 8]
IDS = [c[0] for c in CASES]


def check_hq(dsss, orc, hs, out, pb, seed=3469931):
    n = hs.n
    s = orc.Strings.from_host(hs)
    r = orc.hq_sort(s, pb, seed)
    p = len(pb) - 1
    assert np.array_equal(np.asarray(out["counts"]), r["counts"])
    pw = 1
    while pw * 2 <= p:
        pw *= 2
    assert out["levels"] == pw.bit_length() - 1
    if n == 0:
        return
    lens = u64(out["lengths"], n)
    offs = out["offsets"][:n].cpu().numpy().astype(np.int64)
    chars = out["chars"].cpu().numpy()
    want = [s.get(int(i)) for i in r["source"]]
    got = [chars[o:o + int(l)].tobytes() for o, l in zip(offs, lens)]
    assert got == want
    assert all(chars[o + int(l)] == 0 for o, l in zip(offs, lens))
    assert [s.get(int(i)) for i in u64(out["source"], n)] == want
    assert offs[0] == 0 and np.array_equal(offs[1:], offs[:-1] + lens[:-1].astype(np.int64) + 1)


@pytest.mark.parametrize("p", [1, 2, 3, 8, 13])
@pytest.mark.parametrize("name,strs", CASES, ids=IDS)
def test_hq_sort_matches_oracle(dsss, orc, ctx, name, strs, p):
    hs = host_of(dsss, strs)
    pb = np.linspace(0, hs.n, p + 1).astype(np.uint64)
    out = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), p, part_begin=pb)
    check_hq(dsss, orc, hs, out, pb)


@pytest.mark.parametrize("p", [4, 16, 64])
def test_hq_sort_dn_and_suffixes(dsss, orc, ctx, p):
    for hs in (dsss.gen_dn(40000, 100, 50, seed=p), dsss.gen_suffix_strings(40000, 256, seed=p)):
        pb = dsss.equal_parts(hs.n, p).astype(np.uint64)
        out = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), p, part_begin=pb)
        check_hq(dsss, orc, hs, out, pb)


def test_hq_sort_seeds(dsss, orc, ctx):
    """Equal strings split by the random bits: other seeds, other counts, each
    the oracle's."""
    strs = [b"x"] * 37 + [b"y"] * 29 + [b""] * 11
    hs = host_of(dsss, strs)
    pb = np.array([0, 20, 33, 50, 77], np.uint64)
    seen = set()
    for seed in range(3469931, 3469931 + 12):
        out = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), 4, part_begin=pb, seed=seed)
        check_hq(dsss, orc, hs, out, pb, seed)
        seen.add(tuple(np.asarray(out["counts"]).tolist()))
    assert len(seen) > 1


@pytest.mark.parametrize("strs,pb", [
    ([], [0, 0, 0]),
    ([b"solo"], [0, 1]),
    ([b"b", b"a"], [0, 0, 2]),                      # the first PE is empty: the pivot is ""
    ([b"", b"c", b"a"], [0, 0, 0, 2, 3]),
    ([b"", b"", b"", b""], [0, 1, 4]),              # empty strings only
    ([b"b", b"a", b"c"], [0, 1, 1, 2, 2, 3]),       # p = 5 > n with empty PEs
])
def test_hq_sort_edges(dsss, orc, ctx, strs, pb):
    hs = host_of(dsss, strs)
    pb = np.asarray(pb, np.uint64)
    out = dsss.hq_sort(ctx, dsss.DeviceStrings(hs), len(pb) - 1, part_begin=pb)
    check_hq(dsss, orc, hs, out, pb)
