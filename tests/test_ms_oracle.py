"""The oracle's merge-sort path (oracle_ms_sort), on the CPU: every receiving
PE's output is its received strings in sorted order with their LCPs, the
outputs together are the input once, the interval table adds up, and the
average LCP is getAvgLcp's (the sum of the PEs' local LCP arrays over the
number of strings, integer division)."""
import numpy as np
import pytest

from dist_oracle import pack_list
from inputs import random_strings, run_suffixes, shared_head, with_duplicates


def strings(strs, orc):
    chars, offs, lens, _ = pack_list(strs)
    return orc.Strings(chars, offs.astype(np.uint64), lens.astype(np.uint32))


def lcp_of(a, b):
    m = 0
    while m < len(a) and m < len(b) and a[m] == b[m]:
        m += 1
    return m


CASES = [
    ("random", random_strings(1500, 0, 30, b"ABC", seed=51)),
    ("dups", with_duplicates(random_strings(1200, 0, 20, b"AB", seed=52), 0.3, seed=53)),
    ("shared_head", shared_head(1000, 120, 10, seed=54)),
    ("runs", run_suffixes(seed=55)[:1500]),
]


@pytest.mark.parametrize("p", [1, 3, 8])
@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_ms_oracle_properties(orc, name, strs, p):
    s = strings(strs, orc)
    n = s.n
    pb = np.linspace(0, n, p + 1).astype(np.uint64)
    o = orc.ms_sort(s, pb)
    # the local LCP arrays (0 at each PE start) give the average
    assert o["avg_lcp"] == int(o["lcp"].sum()) // n
    src = o["source"].astype(np.int64)
    assert sorted(src.tolist()) == list(range(n))
    rc = o["recv_counts"].astype(np.int64)
    assert int(rc.sum()) == n
    if p > 1:
        assert np.array_equal(o["intervals"].sum(axis=0).astype(np.int64), rc)
    k = 0
    for r in range(p):
        run = [s.get(int(i)) for i in src[k:k + rc[r]]]
        assert run == sorted(run)
        for j in range(len(run)):
            want = 0 if j == 0 else lcp_of(run[j - 1], run[j])
            assert int(o["out_lcp"][k + j]) == want
        k += rc[r]
    # receiving PEs hold consecutive ranges of the global order
    allstr = [s.get(int(i)) for i in src]
    assert allstr == sorted(allstr)


def truncation_case():
    """p = 2.  PE 0: "00000".."00998", then X = "01000" + "Q"*3000 + "A" and the
    sampled S = "01000" + "Q"*3000 + "B" (local positions 999 and 1000), then
    "01001".."02999"; PE 1: "000000".."002999" (all below PE 0's samples).  The
    average LCP is 4, so samples are cut at 200 * (4 + 5) = 1800 bytes; the one
    splitter is S cut to 1800 bytes, a proper prefix of X, so X (below S but
    above the cut) goes to PE 1: PE 0 sends 999 strings to PE 0, not 1000."""
    pe0 = [b"%05d" % i for i in range(999)]
    pe0 += [b"01000" + b"Q" * 3000 + b"A", b"01000" + b"Q" * 3000 + b"B"]
    pe0 += [b"%05d" % i for i in range(1001, 3000)]
    pe1 = [b"%06d" % i for i in range(3000)]
    return pe0 + pe1, np.array([0, 3000, 6000], np.uint64)


def test_ms_oracle_truncated_splitter(orc):
    strs, pb = truncation_case()
    o = orc.ms_sort(strings(strs, orc), pb)
    assert o["avg_lcp"] == 4
    assert o["intervals"][0].tolist() == [999, 2001]
    assert o["intervals"][1].tolist() == [3000, 0]
