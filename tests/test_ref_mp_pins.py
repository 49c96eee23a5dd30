"""The oracle pinned to the reference itself at p > 1: the reference's own
DistributedPrefixDoublingSort (both samplers), DistributedMergeSort and
RQuick run as real ranks (one process per PE) over the process-based MPI
stand-in (oracle/ref_bridge_mp.cpp, oracle/shim_mpi), compared with the
oracle's single-process restatement on the same strings and PE bounds.  CPU
only; skipped where oracle/_ref was not built."""
import numpy as np
import pytest

from inputs import long_prefix, random_strings, run_suffixes, shared_head, with_duplicates


def strings_of(orc, strs):
    lens = np.array([len(x) for x in strs], np.uint32)
    offs = np.zeros(len(strs), np.uint64)
    if strs:
        offs[1:] = np.cumsum(lens.astype(np.uint64) + 1)[:-1]
    chars = np.frombuffer(b"".join(x + b"\0" for x in strs) + b"\0" * 32, np.uint8).copy()
    return orc.Strings(chars, offs, lens)


def dn_strings(orc, n, L, k, seed, **gk):
    g = orc.gen_dn(n, L, k, seed=seed, **gk)
    return [g.get(i) for i in range(g.n)]


INPUTS = {
    "dups_acgt": lambda orc: with_duplicates(random_strings(3000, 0, 30, b"ACGT", 5)),
    "binary": lambda orc: random_strings(2500, 0, 40, b"AB", 4),
    "long_prefix": lambda orc: long_prefix(1200, 300, 40),
    "shared_head": lambda orc: shared_head(2000),
    "run_suffixes": lambda orc: run_suffixes(max_len=120),
    "dn_rule": lambda orc: dn_strings(orc, 20000, 100, 50, 7),
    "dn_skewed": lambda orc: dn_strings(orc, 6000, 100, 20, 3, long_len=500, long_k=400, frac_long=0.2),
}


@pytest.fixture(scope="module")
def ref_mp(orc):
    if not orc.ref_mp_available():
        pytest.skip("oracle/_ref/ref_mp not built (no reference tree when oracle/ was built)")
    return orc


def parts(n, p, uneven=False):
    if not uneven:
        return np.array([n * q // p for q in range(p + 1)], np.uint64)
    rng = np.random.default_rng(p)
    cut = np.sort(rng.integers(0, n + 1, size=p - 1))
    return np.concatenate([[0], cut, [n]]).astype(np.uint64)


def same_bytes_in_order(s, a, b):
    return [s.get(int(i)) for i in a] == [s.get(int(i)) for i in b]


@pytest.mark.parametrize("name", sorted(INPUTS))
@pytest.mark.parametrize("p,uneven", [(2, False), (3, True), (8, False), (16, True)])
def test_pd_sort_against_reference_ranks(ref_mp, name, p, uneven):
    strs = INPUTS[name](ref_mp)
    s = strings_of(ref_mp, strs)
    pb = parts(s.n, p, uneven)
    res = ref_mp.run_reference_mp("pd", s, pb)
    r = ref_mp.pd_sort(s, pb)
    order = np.concatenate([x["order"] + pb[q] for q, x in enumerate(res)])
    # byte-identical strings have no observable order in radixsort_CI3
    assert same_bytes_in_order(s, order, r["order"])
    assert np.array_equal(np.concatenate([x["lcp"] for x in res]), r["lcp"])
    assert np.array_equal(np.concatenate([x["dp"] for x in res]), r["dp"])
    assert np.array_equal(np.stack([x["intervals"] for x in res]), r["intervals"])
    perm = np.concatenate([x["perm"] for x in res]).reshape(-1, 2)
    assert np.array_equal(perm[:, 0], r["perm_index"])
    assert np.array_equal(perm[:, 1], r["perm_pe"])
    assert [len(x["perm"]) // 2 for x in res] == [int(c) for c in r["recv_counts"]]


@pytest.mark.parametrize("name", ["dups_acgt", "shared_head", "dn_rule"])
@pytest.mark.parametrize("p", [3, 8])
def test_pd_sort_indexed_sampler_against_reference_ranks(ref_mp, name, p):
    s = strings_of(ref_mp, INPUTS[name](ref_mp))
    pb = parts(s.n, p, uneven=True)
    res = ref_mp.run_reference_mp("pdi", s, pb)
    r = ref_mp.pd_sort(s, pb, indexed=True)
    assert np.array_equal(np.stack([x["intervals"] for x in res]), r["intervals"])
    perm = np.concatenate([x["perm"] for x in res]).reshape(-1, 2)
    assert np.array_equal(perm[:, 0], r["perm_index"])
    assert np.array_equal(perm[:, 1], r["perm_pe"])


@pytest.mark.parametrize("name", sorted(INPUTS))
@pytest.mark.parametrize("p", [2, 5, 16])
def test_merge_sort_against_reference_ranks(ref_mp, name, p):
    s = strings_of(ref_mp, INPUTS[name](ref_mp))
    pb = parts(s.n, p, uneven=p == 5)
    res = ref_mp.run_reference_mp("ms", s, pb)
    m = ref_mp.ms_sort(s, pb)
    assert [len(x["lcp"]) for x in res] == [int(c) for c in m["recv_counts"]]
    got = b"".join(bytes(x["bytes"].astype(np.uint8)) for x in res)
    assert got == b"".join(s.get(int(i)) + b"\0" for i in m["source"])
    assert np.array_equal(np.concatenate([x["lcp"] for x in res]), m["out_lcp"])


@pytest.mark.parametrize("name", sorted(INPUTS))
@pytest.mark.parametrize("p", [2, 4, 7, 16])
def test_hq_sort_against_reference_ranks(ref_mp, name, p):
    """RQuick with the hQuicksort executable's seeds (3469931 + rank): every
    PE's sorted strings, so the counts per PE too, equal the oracle's."""
    s = strings_of(ref_mp, INPUTS[name](ref_mp))
    pb = parts(s.n, p, uneven=p == 7)
    res = ref_mp.run_reference_mp("hq", s, pb)
    h = ref_mp.hq_sort(s, pb)
    c = np.concatenate([[0], np.cumsum(h["counts"])]).astype(np.int64)
    for q in range(p):
        exp = b"".join(s.get(int(i)) + b"\0" for i in h["source"][c[q]:c[q + 1]])
        assert bytes(res[q]["bytes"].astype(np.uint8)) == exp


def test_reference_executable_checks_its_own_output(ref_mp, tmp_path):
    """The reference's prefix_doubling executable, as the CPU reference arm runs
    it, on a file of D/N-rule strings: its own --check / --exhaustiveCheck
    (complete and sorted) pass at p = 4, and it reports sorting_overall for
    every iteration."""
    if not ref_mp.ref_exe_available():
        pytest.skip("oracle/_ref/prefix_doubling not built")
    s = ref_mp.gen_dn(50000, 100, 50, seed=1)
    path = str(tmp_path / "in.txt")
    ref_mp.write_lines(s, path)
    times, out = ref_mp.run_reference_pd(path, 4, 2, extra=("--check", "--exhaustiveCheck"))
    assert len(times) == 2 and all(t > 0 for t in times)
    assert "not sorted" not in out and "not complete" not in out
