"""The full path at the benchmark sizes (32e6 strings x 200 B and 1e8 x 100 B,
D/N rule, p = 64), checked through properties that need no oracle run:

  - every PE's local order is a permutation of that PE's strings, strictly
    increasing (these inputs have no two equal strings);
  - every string's distinguishing-prefix length is 72 (the rule puts the
    distinguishing digits at bytes 44-49 and random letters after them, so the
    72-byte round is the first at which every prefix is unique);
  - the merged permutation names every string exactly once, each receiving
    PE's run is strictly increasing, and the merged LCPs are the LCPs of
    neighbours in the run (0 at a run start).

Strictly increasing is decided on the first 72 bytes: every string is
distinguished within them, so two different strings differ there and the
first differing byte orders them.  The checks run on the GPU in chunks."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

W = 72          # bytes compared per string
CHUNK = 1 << 20  # strings per gather


def prefix_bytes(ds, ids):
    """[len(ids), W] uint8: the first W bytes of each string, 0 past its end."""
    offs = ds.offsets[ids]
    lens = ds.lengths[ids].long()
    cols = torch.arange(W, device=ids.device)
    b = ds.chars[offs[:, None] + cols[None, :]]
    return torch.where(cols[None, :] < lens[:, None], b, torch.zeros_like(b))


def pair_check(ds, ids, same_run):
    """For neighbours (ids[i], ids[i + 1]) with same_run[i]: strictly
    increasing on the first W bytes; returns their LCPs (int64, -1 where
    same_run is False)."""
    m = ids.numel()
    lcp = torch.full((max(m - 1, 0),), -1, dtype=torch.int64, device=ids.device)
    for s in range(0, m - 1, CHUNK):
        e = min(m - 1, s + CHUNK)
        a = prefix_bytes(ds, ids[s:e])
        b = prefix_bytes(ds, ids[s + 1:e + 1])
        diff = a != b
        run = same_run[s:e]
        assert bool(diff.any(dim=1)[run].all()), "two neighbours share their first 72 bytes"
        first = diff.int().argmax(dim=1)
        av = a.gather(1, first[:, None]).squeeze(1)
        bv = b.gather(1, first[:, None]).squeeze(1)
        assert bool((av < bv)[run].all()), "a neighbour pair is out of order"
        lcp[s:e] = torch.where(run, first.long(), torch.full_like(first.long(), -1))
    return lcp


@pytest.mark.parametrize("n,length", [(32_000_000, 200), (100_000_000, 100)])
def test_full_size_properties(dsss, ctx, n, length):
    p = 64
    hs = dsss.gen_dn(n, length, 50, seed=1)
    ds = dsss.DeviceStrings(hs)
    del hs
    out = dsss.pd_sort(ctx, ds, p)
    dev = ds.offsets.device
    pb = torch.from_numpy(np.asarray(out["part_begin"], np.int64)).to(dev)

    # distinguishing prefixes
    dp = out["dp"][:n].long()
    assert bool((dp == 72).all())

    # local orders: permutation of each PE's id range, strictly increasing inside a PE
    lo = out["local_order"][:n].long() & 0xFFFFFFFF
    pos_pe = torch.repeat_interleave(torch.arange(p, device=dev), pb[1:] - pb[:-1])
    assert bool((torch.searchsorted(pb, lo, right=True) - 1 == pos_pe).all())
    assert bool((torch.sort(lo).values == torch.arange(n, device=dev)).all())
    pair_check(ds, lo, pos_pe[:-1] == pos_pe[1:])

    # merged sequences: ids, one run per receiving PE
    pi = out["perm_index"][:n].long() & 0xFFFFFFFF
    pp = out["perm_pe"][:n].long() & 0xFFFFFFFF
    ids = lo[pb[pp] + pi]
    assert bool((torch.sort(ids).values == torch.arange(n, device=dev)).all())
    rc = torch.from_numpy(np.asarray(out["recv_counts"], np.int64)).to(dev)
    assert int(rc.sum()) == n
    run = torch.repeat_interleave(torch.arange(p, device=dev), rc)
    same = run[:-1] == run[1:]
    lcp = pair_check(ds, ids, same)
    ml = out["merged_lcp"][:n].long() & 0xFFFFFFFF
    starts = torch.ones(n, dtype=torch.bool, device=dev)
    starts[1:] = ~same
    assert bool((ml[starts] == 0).all())
    assert bool((ml[1:][same] == lcp[same]).all())


class _View:
    """chars / offsets / lengths tensors shaped like DeviceStrings."""

    def __init__(self, chars, offsets, lengths):
        self.chars, self.offsets, self.lengths = chars, offsets, lengths


def test_full_size_ms_sort(dsss, ctx):
    """The merge-sort path on 32e6 strings x 200 B, p = 64: the output names
    every string once, each receiving PE's strings are strictly increasing,
    their bytes are the input strings', and the LCPs are the neighbours'."""
    n, p = 32_000_000, 64
    hs = dsss.gen_dn(n, 200, 50, seed=2)
    ds = dsss.DeviceStrings(hs)
    del hs
    out = dsss.ms_sort(ctx, ds, p)
    dev = ds.offsets.device
    src = out["source"][:n].long() & 0xFFFFFFFF
    assert bool((torch.sort(src).values == torch.arange(n, device=dev)).all())
    lens = out["lengths"][:n].long() & 0xFFFFFFFF
    assert bool((lens == ds.lengths[src].long()).all())
    view = _View(out["chars"], out["offsets"][:n], out["lengths"][:n])
    ids = torch.arange(n, device=dev)
    # output bytes equal the input strings' (first W bytes, chunk by chunk)
    for s in range(0, n, CHUNK):
        e = min(n, s + CHUNK)
        assert bool((prefix_bytes(view, ids[s:e]) == prefix_bytes(ds, src[s:e])).all())
    rc = torch.from_numpy(np.asarray(out["recv_counts"], np.int64)).to(dev)
    assert int(rc.sum()) == n
    run = torch.repeat_interleave(torch.arange(p, device=dev), rc)
    same = run[:-1] == run[1:]
    lcp = pair_check(view, ids, same)
    ml = out["lcp"][:n].long() & 0xFFFFFFFF
    starts = torch.ones(n, dtype=torch.bool, device=dev)
    starts[1:] = ~same
    assert bool((ml[starts] == 0).all())
    assert bool((ml[1:][same] == lcp[same]).all())


def test_full_size_hq_sort(dsss, ctx):
    """hQuicksort on 32e6 strings x 200 B, p = 64: the counts add up to n, the
    output names every string once, is strictly increasing across all PEs
    (the PEs in rank order are the global order), and its bytes are the input
    strings'."""
    n, p = 32_000_000, 64
    hs = dsss.gen_dn(n, 200, 50, seed=3)
    ds = dsss.DeviceStrings(hs)
    del hs
    out = dsss.hq_sort(ctx, ds, p)
    dev = ds.offsets.device
    cnt = np.asarray(out["counts"], np.int64)
    assert int(cnt.sum()) == n and out["levels"] == 6
    src = out["source"][:n].long() & 0xFFFFFFFF
    assert bool((torch.sort(src).values == torch.arange(n, device=dev)).all())
    lens = out["lengths"][:n].long() & 0xFFFFFFFF
    assert bool((lens == ds.lengths[src].long()).all())
    view = _View(out["chars"], out["offsets"][:n], out["lengths"][:n])
    ids = torch.arange(n, device=dev)
    for s in range(0, n, CHUNK):
        e = min(n, s + CHUNK)
        assert bool((prefix_bytes(view, ids[s:e]) == prefix_bytes(ds, src[s:e])).all())
    pair_check(view, ids, torch.ones(n - 1, dtype=torch.bool, device=dev))
