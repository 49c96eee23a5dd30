"""The distributed path with the CUDA backend: two or three ranks, each with
its own context on the one GPU, exchanging through gloo (host memory); the
ranks' kernels never wait on one another.  Checked against the oracle's
single-process run of the whole input, as test_dist.py checks the host
backend."""
import pytest

from inputs import random_strings, run_suffixes, shared_head, with_duplicates
from test_dist import check_against_oracle, run_ranks

pytestmark = pytest.mark.gpu


def gen_inputs():
    import __graft_entry__
    d = __graft_entry__.load_package()
    dn = d.gen_dn(12000, 60, 30, seed=7)
    return [
        ("dn", [dn.get(i) for i in range(dn.n)]),
        ("dups", with_duplicates(random_strings(4000, 0, 24, b"ABC", seed=52), 0.3, seed=53)),
        ("shared_head", shared_head(3000, 200, 12, seed=54)),
        ("runs", run_suffixes(seed=55)),
    ]


CASES = gen_inputs()


@pytest.mark.parametrize("sampler", [0, 2])
@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_gpu_ranks_match_oracle(orc, name, strs, sampler):
    n = len(strs)
    pb = [0, n // 9, n // 3, n // 2, (5 * n) // 6, n]
    res = run_ranks(2, (strs, pb, [0, 3, 5], sampler), "gpu")
    check_against_oracle(orc, strs, pb, res, sampler, exact_ties=False)


def test_gpu_three_ranks(orc):
    strs = CASES[0][1]
    n = len(strs)
    pb = [0, n // 4, n // 2, (3 * n) // 4, n]
    res = run_ranks(3, (strs, pb, [0, 1, 3, 4], 0), "gpu")
    check_against_oracle(orc, strs, pb, res, 0, exact_ties=False)


def test_nccl_single_rank(orc):
    """The NCCL code path of the collectives (payloads stay on the GPU), with
    one rank holding all five PEs."""
    strs = CASES[1][1]
    n = len(strs)
    pb = [0, n // 5, (2 * n) // 5, (3 * n) // 5, (4 * n) // 5, n]
    res = run_ranks(1, (strs, pb, [0, 5], 0), "gpu", pg="nccl")
    check_against_oracle(orc, strs, pb, res, 0, exact_ties=False)


@pytest.mark.parametrize("name,strs", CASES, ids=[c[0] for c in CASES])
def test_gpu_ranks_merge_sort(orc, name, strs):
    """DistributedMergeSort with the CUDA backend (dsss_lcp_merge_strings on
    the receiving side): every output string and LCP as the oracle's."""
    from test_dist import check_ms_against_oracle
    n = len(strs)
    pb = [0, n // 9, n // 3, n // 2, (5 * n) // 6, n]
    res = run_ranks(2, (strs, pb, [0, 3, 5], 0, False, "ms"), "gpu")
    check_ms_against_oracle(orc, strs, pb, res)


def test_nccl_single_rank_merge_sort(orc):
    from test_dist import check_ms_against_oracle
    strs = CASES[0][1]
    n = len(strs)
    pb = [0, n // 5, (2 * n) // 5, (3 * n) // 5, (4 * n) // 5, n]
    res = run_ranks(1, (strs, pb, [0, 5], 0, True, "ms"), "gpu", pg="nccl")
    check_ms_against_oracle(orc, strs, pb, res)


def test_gpu_ranks_golomb_coded_hashes(orc):
    """The Golomb/delta-coded hash exchange with the CUDA backend: records
    sorted by dsss_hash_sort, blocks by dsss_golomb_encode, read back by
    dsss_golomb_decode on the owning rank; results equal the oracle's."""
    strs = CASES[1][1]
    n = len(strs)
    pb = [0, n // 6, n // 3, n // 2, (3 * n) // 4, n]
    res = run_ranks(2, (strs, pb, [0, 3, 5], 0, False, "pd", True), "gpu")
    check_against_oracle(orc, strs, pb, res, 0, exact_ties=False)

