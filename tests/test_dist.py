"""The distributed path (dist.py) on CPU ranks over gloo, with the host
backend: collectives, routing of hashes, sample gathering, container exchange
and regrouping, checked against the oracle's single-process run of the whole
input.  test_gpu_dist.py runs the same flow with the CUDA backend."""
import os
import socket
import tempfile

import numpy as np
import pytest

from inputs import random_strings, run_suffixes, shared_head, with_duplicates


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world, inputs, backend, pg="gloo"):
    import torch.multiprocessing as mp
    from dist_worker import rank_main
    with tempfile.TemporaryDirectory() as tmp:
        mp.spawn(rank_main, args=(world, free_port(), tmp, inputs, backend, pg), nprocs=world, join=True)
        return [dict(np.load(os.path.join(tmp, f"rank{r}.npz"))) for r in range(world)]


def check_against_oracle(orc, strs, pb, results, sampler, exact_ties=True):
    from dist_oracle import pack_list
    chars, offs, lens, _ = pack_list(strs)
    s = orc.Strings(chars, offs.astype(np.uint64), lens.astype(np.uint32))
    ref = orc.pd_sort(s, np.asarray(pb, np.uint64), indexed=sampler == 2)
    p = len(pb) - 1
    rb = np.concatenate([[0], np.cumsum(ref["recv_counts"])]).astype(np.int64)
    for r in results:
        q0, q1, s0 = int(r["q0"]), int(r["q1"]), int(r["s0"])
        s1 = int(pb[q1])
        assert np.array_equal(r["local_order"] + s0, ref["order"][s0:s1].astype(np.int64))
        if p == 1:
            continue
        assert np.array_equal(r["dp"], ref["dp"][s0:s1].astype(np.int64))
        assert np.array_equal(r["intervals"], ref["intervals"][q0:q1].astype(np.int64))
        assert np.array_equal(r["recv_counts"], ref["recv_counts"][q0:q1].astype(np.int64))
        b0, b1 = rb[q0], rb[q1]
        gi, gp = r["perm_index"], r["perm_pe"]
        ri, rp = ref["perm_index"][b0:b1].astype(np.int64), ref["perm_pe"][b0:b1].astype(np.int64)
        assert np.array_equal(r["merged_lcp"], ref["merged_lcp"][b0:b1].astype(np.int64))
        if exact_ties:
            assert np.array_equal(gi, ri) and np.array_equal(gp, rp)
        else:
            assert sorted(zip(gp.tolist(), gi.tolist())) == sorted(zip(rp.tolist(), ri.tolist()))


def cases():
    a = random_strings(1500, 0, 30, b"ABC", seed=41)
    b = with_duplicates(random_strings(1200, 0, 20, b"AB", seed=42), 0.3, seed=43)
    c = shared_head(1000, 120, 10, seed=44)
    d = run_suffixes(seed=45)[:1500]
    return [("random", a), ("dups", b), ("shared_head", c), ("runs", d)]


CASES = cases()


@pytest.mark.parametrize("sampler", [0, 2])
@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_two_ranks_match_oracle(orc, name, strs, sampler):
    n = len(strs)
    pb = [0, n // 7, n // 3, n // 2, (4 * n) // 5, n]          # 5 PEs of uneven sizes
    splits = [0, 2, 5]                                        # rank 0: PEs 0-1, rank 1: PEs 2-4
    res = run_ranks(2, (strs, pb, splits, sampler), "oracle")
    check_against_oracle(orc, strs, pb, res, sampler)


@pytest.mark.parametrize("name,strs", CASES[:2] + CASES[3:], ids=["random", "dups", "runs"])
def test_two_ranks_compressed_lcps(orc, name, strs):
    """compressLcps: the LCPs cross as varint bytes; results unchanged."""
    n = len(strs)
    pb = [0, n // 4, n // 2, (3 * n) // 4, n]
    res = run_ranks(2, (strs, pb, [0, 1, 4], 0, True), "oracle")
    check_against_oracle(orc, strs, pb, res, 0)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name,strs", CASES[:2] + CASES[3:], ids=["random", "dups", "runs"])
def test_golomb_coded_hashes(orc, name, strs, world):
    """sequentialGolombEncoding: every round's hashes cross sorted and
    Golomb/delta-coded, one block per owning rank; results unchanged."""
    n = len(strs)
    pb = [0, n // 5, n // 3, n // 2, (3 * n) // 4, n]
    splits = [0, 2, 5] if world == 2 else [0, 1, 3, 5]
    res = run_ranks(world, (strs, pb, splits, 0, False, "pd", True), "oracle")
    check_against_oracle(orc, strs, pb, res, 0)


def test_three_ranks_one_pe_each(orc):
    strs = CASES[0][1]
    n = len(strs)
    pb = [0, n // 3, (2 * n) // 3, n]
    res = run_ranks(3, (strs, pb, [0, 1, 2, 3], 0), "oracle")
    check_against_oracle(orc, strs, pb, res, 0)


def test_pack_rows_round_trip(dsss):
    """The one-message packing of the sample all-gather: columns of any
    length (empty too) and a byte blob of any length come back unchanged."""
    from dsss_b200 import dist
    rng = np.random.default_rng(3)
    for ncols, nb in ((3, 0), (3, 1), (3, 13), (1, 64), (0, 5)):
        cols = [rng.integers(-2**40, 2**40, size=int(rng.integers(0, 9)), dtype=np.int64) for _ in range(ncols)]
        if ncols:
            cols[0] = np.zeros(0, np.int64)
        blob = rng.integers(0, 256, size=nb, dtype=np.uint8)
        got, gb = dist._unpack_rows(dist._pack_rows(*cols, blob=blob))
        assert len(got) == ncols
        for a, b in zip(cols, got):
            assert np.array_equal(a, b)
        assert np.array_equal(gb, blob)


def test_sample_positions_match_reference_rule(dsss):
    """floor(i * (n_q / (nr + 1))) in double arithmetic for i = 1..nr."""
    from dsss_b200 import dist
    for nq, p in ((0, 4), (1, 4), (5, 4), (1000, 64), (999_999, 64), (7, 2)):
        nr = min(2 * (p - 1), nq)
        want = [int(float(i) * (float(nq) / float(nr + 1))) for i in range(1, nr + 1)]
        assert dist.sample_positions([nq], p)[0].tolist() == want


def check_ms_against_oracle(orc, strs, pb, results):
    """DistributedMergeSort over ranks against the oracle's single-process
    merge-sort path: average LCP, local orders, interval rows, strings per
    receiving PE, every output string's bytes and its LCP."""
    from dist_oracle import pack_list
    chars, offs, lens, _ = pack_list(strs)
    s = orc.Strings(chars, offs.astype(np.uint64), lens.astype(np.uint32))
    ref = orc.ms_sort(s, np.asarray(pb, np.uint64))
    rb = np.concatenate([[0], np.cumsum(ref["recv_counts"])]).astype(np.int64)
    for r in results:
        q0, q1, s0 = int(r["q0"]), int(r["q1"]), int(r["s0"])
        s1 = int(pb[q1])
        assert int(r["avg_lcp"]) == ref["avg_lcp"]
        assert np.array_equal(r["local_order"] + s0, ref["order"][s0:s1].astype(np.int64))
        assert np.array_equal(r["intervals"], ref["intervals"][q0:q1].astype(np.int64))
        assert np.array_equal(r["recv_counts"], ref["recv_counts"][q0:q1].astype(np.int64))
        b0, b1 = rb[q0], rb[q1]
        oc, oo, ol = r["out_chars"], r["out_offsets"], r["out_lengths"]
        got = [oc[o:o + l].tobytes() for o, l in zip(oo, ol)]
        assert got == [s.get(int(i)) for i in ref["source"][b0:b1]]
        assert np.array_equal(r["out_lcp"], ref["out_lcp"][b0:b1].astype(np.int64))


@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_two_ranks_merge_sort(orc, name, strs):
    n = len(strs)
    pb = [0, n // 7, n // 3, n // 2, (4 * n) // 5, n]
    res = run_ranks(2, (strs, pb, [0, 2, 5], 0, False, "ms"), "oracle")
    check_ms_against_oracle(orc, strs, pb, res)


def test_merge_sort_compressed_lcps_three_ranks(orc):
    """Three ranks, one with no PE's strings in its first PE, LCPs sent as
    varint bytes."""
    strs = CASES[1][1]
    n = len(strs)
    pb = [0, 0, n // 3, (2 * n) // 3, n]
    res = run_ranks(3, (strs, pb, [0, 2, 3, 4], 0, True, "ms"), "oracle")
    check_ms_against_oracle(orc, strs, pb, res)


@pytest.mark.parametrize("mode", ["pd", "ms"])
def test_rank_without_pes(orc, mode):
    """Rank 0 holds no PE: it still takes part in every collective."""
    strs = CASES[0][1]
    n = len(strs)
    pb = [0, n // 3, (2 * n) // 3, n]
    res = run_ranks(2, (strs, pb, [0, 0, 3], 0, False, mode), "oracle")
    if mode == "ms":
        check_ms_against_oracle(orc, strs, pb, res)
    else:
        check_against_oracle(orc, strs, pb, res, 0)
