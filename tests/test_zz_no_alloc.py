"""dsss_adjacent_lcp_noalloc — the entry point for callers that cannot
allocate device memory (inside another framework's memory pool, or in loops
that cannot take cudaMalloc's device-wide synchronisation).  Its output must
equal the allocating dsss_adjacent_lcp's on the same input, call after call
(the static scratch it reuses keeps the previous call's contents)."""
import numpy as np
import pytest
import torch

from inputs import long_prefix, random_strings

pytestmark = pytest.mark.gpu


def sorted_ids(orc, hs):
    order, _ = orc.local_sort(orc.Strings.from_host(hs), np.array([0, hs.n], np.uint64))
    return torch.from_numpy(order.astype(np.int32)).cuda()


def test_noalloc_matches_allocating_entry_two_calls(dsss, orc, ctx):
    # Two different inputs in a row; both have neighbours sharing more than
    # 64 bytes, so the scratch queue of the warp pass is used each time.
    inputs = [
        dsss.from_bytes_list(long_prefix(3000, 600, 40, 91) + random_strings(2000, 0, 80, b"AB", 92)),
        dsss.from_bytes_list(long_prefix(5000, 130, 10, 93)),
    ]
    for hs in inputs:
        ds = dsss.DeviceStrings(hs)
        order = sorted_ids(orc, hs)
        want = dsss.adjacent_lcp(ctx, ds, order)
        got = torch.full((hs.n,), -1, dtype=torch.int32, device="cuda")
        dsss.adjacent_lcp_noalloc(ds, order, got)
        torch.cuda.synchronize()
        assert torch.equal(got, want)  # integer LCPs: exact


def test_noalloc_rejects_too_many_strings(dsss):
    hs = dsss.from_bytes_list([b"A", b"B"])
    ds = dsss.DeviceStrings(hs)
    big = (1 << 22) + 1
    order = torch.zeros(1, dtype=torch.int32, device="cuda")
    lcp = torch.zeros(1, dtype=torch.int32, device="cuda")
    import ctypes
    rc = dsss.lib().dsss_adjacent_lcp_noalloc(ctypes.byref(ds.arena()), order.data_ptr(), big, lcp.data_ptr(),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -22
    assert b"at most" in dsss.lib().dsss_last_error()
