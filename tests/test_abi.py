"""The C ABI library loads and exports every entry point include/dsss.h
declares; host-only entry points (generators) work without a GPU; device
entry points fail loudly when there is no GPU.  CPU only."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    with open(os.path.join(ROOT, "include", "dsss.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|uint64_t|double|const char\*)\s+(dsss_\w+)\s*\(", src, re.M)))


def test_header_symbols_exported(dsss):
    import ctypes
    lib = ctypes.CDLL(dsss.LIB_PATH)
    names = declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(dsss.exported_symbols()) | {"dsss_abi_version"}


def test_abi_version(dsss):
    assert dsss.lib().dsss_abi_version() == 1


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly(dsss):
    with pytest.raises(dsss.DsssError) as e:
        dsss.Context(0)
    assert e.value.code == -5


def test_library_is_sm100a_only():
    """libdsss.so carries sm_100a code only (cuobjdump is not used: the build
    command is checked instead)."""
    with open(os.path.join(ROOT, "distributed-string-sorting_b200", "build.py")) as f:
        src = f.read()
    assert "arch=compute_100a,code=sm_100a" in src


def compute_D(strs_sorted):
    """D as DNGenerator_tests.cpp:22-45 defines it: sum of max(lcp with
    neighbours) + 1 over the sorted set."""
    n = len(strs_sorted)
    if n < 2:
        return 0
    lcps = [0] * n
    for i in range(1, n):
        a, b = strs_sorted[i - 1], strs_sorted[i]
        m = 0
        while m < min(len(a), len(b)) and a[m] == b[m]:
            m += 1
        lcps[i] = m
    D = sum(max(lcps[i], lcps[i + 1]) + 1 for i in range(n - 1)) + lcps[-1] + 1
    return D


@pytest.mark.parametrize("n,L,k", [(1000, 100, 50), (10000, 250, 125), (20000, 500, 50)])
def test_dn_generator_ratio(dsss, n, L, k):
    """DNGenerator_tests.cpp:47-104: D/N of the generated set matches the
    requested ratio k/L (within 0.01 of the string length ratio)."""
    hs = dsss.gen_dn(n, L, k, seed=3)
    strs = sorted(hs.get(i) for i in range(n))
    D = compute_D(strs)
    N = sum(len(s) for s in strs)
    assert abs(D / N - k / L) < 0.01, (D / N, k / L)


def test_dn_generator_layout_and_seed(dsss):
    a = dsss.gen_dn(5000, 60, 30, seed=5)
    b = dsss.gen_dn(5000, 60, 30, seed=5)
    c = dsss.gen_dn(5000, 60, 30, seed=6)
    assert np.array_equal(a.chars, b.chars) and not np.array_equal(a.chars, c.chars)
    assert np.all(a.lengths == 60)
    assert np.all(a.chars[a.offsets + 60] == 0)
    strs = [a.get(i) for i in range(a.n)]
    assert len(set(strs)) == a.n  # unique digits make every string distinct
    assert all(s[:30 - 3] == b"A" * 27 for s in strs)  # 30 - ceil(log26 5000) filler 'A's


def test_skewed_generator(dsss):
    hs = dsss.gen_dn(50000, 100, 20, seed=2, long_len=500, long_k=400, frac_long=0.2)
    frac = float(np.mean(hs.lengths == 500))
    assert abs(frac - 0.2) < 0.01
    assert set(np.unique(hs.lengths).tolist()) == {100, 500}


def test_suffix_generator(dsss):
    hs = dsss.gen_suffix_strings(100000, 256, seed=3)
    assert hs.n == 100000
    assert int(hs.lengths.max()) == 256 and int(hs.lengths[-1]) == 1
    assert set(np.unique(hs.chars[:100000]).tolist()) <= set(b"ACGT")
    # copied blocks make long repeats: many 256-byte suffixes occur more than once
    strs = [hs.get(i) for i in range(0, 100000 - 256, 7)]
    assert len(set(strs)) < len(strs)


def test_request_generator(dsss):
    hs = dsss.gen_request(20000, seed=4)
    assert hs.lengths.min() >= 8 and hs.lengths.max() <= 256
    assert 40 < float(hs.lengths.mean()) < 80
    body = np.concatenate([hs.chars[int(o):int(o) + int(l)] for o, l in zip(hs.offsets[:200], hs.lengths[:200])])
    assert body.min() >= 0x21 and body.max() <= 0x7E


def test_knob_errors(dsss):
    """Tuning knobs are host state: set, read back, range-checked, reset."""
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("no_such_knob", 1)
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("sort_small_max", 100000)
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("merge_extend_lanes", 3)
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("merge_extend_lanes", 2)
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("copy_word", 12)
    assert dsss.tune_get("copy_word") == 16
    v = dsss.tune_get("dp_filter_bits")
    dsss.tune_set("dp_filter_bits", 8)
    assert dsss.tune_get("dp_filter_bits") == 8
    dsss.tune_set("dp_filter_bits", -1)
    assert dsss.tune_get("dp_filter_bits") == v == 16


def test_digit_knobs(dsss):
    """The MSD digit knobs: bit digits over the arena 0 / 1 / 2 / 3 and inside the
    segment sorter 0 / 1, both off by default; every knob the package lists
    can be read."""
    assert dsss.tune_get("sort_bits") == 0 and dsss.tune_get("sort_seg_bits") == 0
    for v in (1, 2, 3, 0):
        dsss.tune_set("sort_bits", v)
        assert dsss.tune_get("sort_bits") == v
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("sort_bits", 4)
    with pytest.raises(dsss.DsssError):
        dsss.tune_set("sort_seg_bits", 2)
    dsss.tune_set("sort_seg_bits", 1)
    assert dsss.tune_get("sort_seg_bits") == 1
    dsss.tune_set("sort_seg_bits", -1)
    dsss.tune_set("sort_bits", -1)
    assert dsss.tune_get("sort_bits") == 0 and dsss.tune_get("sort_seg_bits") == 0
    for name in dsss.TUNE_KNOBS:
        dsss.tune_get(name)
