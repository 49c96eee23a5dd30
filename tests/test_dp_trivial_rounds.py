"""Why the GPU may leave out the first distinguishing-prefix rounds.  It
skips a round while every string is still a candidate and the round's depth
is at most both the shortest string and T = min over sorted positions of
max(lcp[i], lcp[i + 1]), with lcp[0] and lcp[n] taken as 0.  In such a round
every string is an LCP-local duplicate or a root, so every string stays.
The oracle runs every round (BloomFilter::filter as the reference does,
bloomfilter.hpp:1415-1556), so its per-round candidate counts must be n for
those rounds.  Checked here on the CPU, with one PE, whose local order is
the global order that the GPU's rounds run over."""
import numpy as np
import pytest

from dist_oracle import pack_list
from inputs import cases, long_prefix, random_strings, shared_head, with_duplicates


def strings(strs, orc):
    chars, offs, lens, _ = pack_list(strs)
    return orc.Strings(chars, offs.astype(np.uint64), lens.astype(np.uint32))


def depths(k):
    return [8] + [8 + (16 << j) for j in range(k - 1)]


def families():
    out = [(name, s) for name, s in cases() if len(s) >= 2]
    out += [("long_prefix", long_prefix(3000, 44, 30)),
            ("long_prefix_dups", with_duplicates(long_prefix(3000, 100, 8), 0.2)),
            ("shared_head", shared_head(2000)),
            ("ab", random_strings(3000, 20, 60, b"AB", seed=5))]
    return out


@pytest.mark.parametrize("name,strs", families(), ids=[f[0] for f in families()])
def test_rounds_up_to_the_lcp_bound_keep_every_string(orc, name, strs):
    s = strings(strs, orc)
    n = s.n
    pb = np.array([0, n], np.uint64)
    order, lcp = orc.local_sort(s, pb)
    lcp = np.asarray(lcp, np.int64)
    nbr = np.maximum(np.where(np.arange(n) > 0, lcp, 0), np.append(lcp[1:], 0))
    bound = min(int(nbr.min()), min(len(x) for x in strs))
    dp, counts = orc.dp_rounds(s, pb, order, lcp.astype(np.uint64))
    skipped = 0
    for r, d in enumerate(depths(len(counts))):
        if d > bound:
            break
        assert int(counts[r]) == n, (name, d, bound)
        skipped += 1
    if name.startswith("long_prefix"):  # strings sharing 44 or 100 bytes: rounds 8, 24, 40 at least
        assert skipped >= 3
