"""Device-side generators: the benchmark inputs made in HBM are byte for byte
the host generators' (and, for the D/N rule, the oracle's own restatement of
the rule), so a configuration's strings need not cross PCIe."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_view(ds):
    n = ds.n
    return (ds.chars[:ds.char_bytes].cpu().numpy(), ds.offsets[:n].cpu().numpy().view(np.uint64),
            ds.lengths[:n].cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("n,L,k,gk", [
    (1, 10, 5, {}),
    (1000, 100, 50, {}),
    (200_000, 200, 50, {}),
    (300_000, 100, 20, dict(long_len=500, long_k=400, frac_long=0.2)),
    (50_000, 7, 7, {}),  # records shorter than a 16-byte word
    (70_000, 30, 10, dict(long_len=40, long_k=20, frac_long=0.5)),
])
def test_dn_device_equals_oracle(dsss, orc, ctx, n, L, k, gk):
    ds = dsss.gen_dn_device(ctx, n, L, k, seed=9, **gk)
    ref = orc.gen_dn(n, L, k, seed=9, **gk)
    chars, offs, lens = host_view(ds)
    assert ds.char_bytes == ref.char_bytes
    assert np.array_equal(chars, ref.chars[:ref.char_bytes])
    assert np.array_equal(offs, ref.offsets)
    assert np.array_equal(lens, ref.lengths)


def test_dn_device_sorts_like_host(dsss, orc, ctx):
    """A device-generated set through the full path: the oracle's result."""
    from test_gpu_parity import check_pd
    ds = dsss.gen_dn_device(ctx, 60_000, 100, 50, seed=4)
    out = dsss.pd_sort(ctx, ds, 8)
    check_pd(dsss, orc, dsss.gen_dn(60_000, 100, 50, seed=4), out, 8)


@pytest.mark.parametrize("n", [1, 5000, 400_000])
def test_request_device_equals_host(dsss, ctx, n):
    ds = dsss.gen_request_device(ctx, n, seed=77)
    h = dsss.gen_request(n, seed=77)
    chars, offs, lens = host_view(ds)
    assert ds.char_bytes == h.char_bytes
    assert np.array_equal(chars, h.chars[:h.char_bytes])
    assert np.array_equal(offs, h.offsets)
    assert np.array_equal(lens, h.lengths)


def test_suffix_views_device_equal_host(dsss):
    ds = dsss.gen_suffix_strings_device(1 << 20, 256, seed=5)
    h = dsss.gen_suffix_strings(1 << 20, 256, seed=5)
    chars, offs, lens = host_view(ds)
    assert np.array_equal(chars, h.chars[:h.char_bytes])
    assert np.array_equal(offs, h.offsets)
    assert np.array_equal(lens, h.lengths)
