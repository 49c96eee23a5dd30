"""Varint coding of LCP arrays on the GPU (dsss_varint_encode / _decode)
against the restatement of Writer::PutVarint / writeRanges: the same bytes,
the same per-range byte counts, and the values back; malformed input is
rejected.  Then the distributed path with compressed LCPs on the GPU backend."""
import numpy as np
import pytest
import torch

from test_dist import CASES, check_against_oracle, run_ranks

pytestmark = pytest.mark.gpu


def values(seed, n):
    rng = np.random.default_rng(seed)
    # every size class: 1 to 5 bytes
    bits = rng.integers(0, 33, size=n)
    v = (rng.integers(0, 2**32, size=n, dtype=np.uint64) >> (32 - bits).astype(np.uint64)).astype(np.uint64)
    edge = np.array([0, 127, 128, 16383, 16384, 2**32 - 1], np.uint64)
    v[:min(n, 6)] = edge[:min(n, 6)]
    return v


@pytest.mark.parametrize("n,ranges", [(0, [0, 0]), (1, [1]), (1000, [300, 0, 700]), (200000, [50000] * 4)])
def test_varint_matches_reference_format(dsss, orc, ctx, n, ranges):
    v = values(n + 7, n)
    dv = torch.from_numpy(v.astype(np.uint32).view(np.int32)).cuda()
    got, per = dsss.varint_encode(ctx, dv, ranges)
    want, wper = orc.varint_encode(v, ranges)
    assert np.array_equal(got.cpu().numpy(), want)
    assert np.array_equal(per, wper)
    back = dsss.varint_decode(ctx, got, n)
    assert np.array_equal(back.cpu().numpy().view(np.uint32).astype(np.uint64), v)


def test_varint_decode_rejects_bad_input(dsss, ctx):
    cut = torch.tensor([0x81, 0x82], dtype=torch.uint8, device="cuda")          # last value cut off
    with pytest.raises(dsss.DsssError):
        dsss.varint_decode(ctx, cut, 1)
    long6 = torch.tensor([0x80] * 5 + [0x01], dtype=torch.uint8, device="cuda")  # 6 bytes
    with pytest.raises(dsss.DsssError):
        dsss.varint_decode(ctx, long6, 1)
    two = torch.tensor([0x01, 0x02], dtype=torch.uint8, device="cuda")          # 2 values, not 3
    with pytest.raises(dsss.DsssError):
        dsss.varint_decode(ctx, two, 3)


def test_dist_gpu_compressed_lcps(orc):
    """Two ranks (gloo) on the CUDA backend with compressLcps."""
    strs = CASES[1][1]
    n = len(strs)
    pb = [0, n // 4, n // 2, (3 * n) // 4, n]
    res = run_ranks(2, (strs, pb, [0, 1, 4], 0, True), "gpu")
    check_against_oracle(orc, strs, pb, res, 0, exact_ties=False)


def test_varint_encode_rejects_ranges_not_starting_at_zero(dsss, ctx):
    """range_begin must start at 0: a first bound past 0 would leave values
    before it coded but counted in no range."""
    import ctypes
    v = torch.arange(8, dtype=torch.int32, device="cuda")
    rb = np.array([1, 5, 8], np.uint64)
    tot = ctypes.c_uint64(0)
    per = np.zeros(2, np.uint64)
    rc = dsss.lib().dsss_varint_encode(ctx.h, v.data_ptr(), 8, rb.ctypes.data, 2, None, 0, ctypes.byref(tot),
                                       per.ctypes.data, None)
    assert rc == -22  # DSSS_EINVAL
