"""bench.py's roofline arithmetic on the CPU: every kernel with a byte
formula has its per-step bytes and a traffic entry, and pd_rooflines turns
event times into achieved GB/s and fractions of the peak as stated
(algorithmic bytes over the kernel's summed event time)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_formula_tables_agree():
    assert set(bench.DRAM_PER_UNIT) >= set(bench.ROOFLINE_BYTES)


def test_pd_rooflines_arithmetic():
    torch = pytest.importorskip("torch")
    n, L = 1000, 200
    dp = torch.full((n,), 72, dtype=torch.int32)
    lcp = torch.full((n,), 50, dtype=torch.int32)
    out = {"dp": dp, "merged_lcp": lcp}
    steps = 2
    # (launches, total ms) over the steps, as Context.kernel_times reports
    kt = {"k_prefix": (4, 0.02), "k_scatter": (8, 0.03), "k_bucket_direct": (2, 0.004),
          "stage:sort": (2, 0.06), "stage:merge": (2, 0.01)}
    r = bench.pd_rooflines(out, np.full(n, L, np.uint32), n, kt, steps, 1000.0, "measured")
    rp = r["rooflines"]["k_prefix"]
    algo = (72 + 36) * n
    assert rp["algo_bytes"] == algo
    assert rp["kernel_ms"] == pytest.approx(0.01)
    assert rp["achieved"] == pytest.approx(algo / 1e-5 / 1e9)
    assert rp["frac"] == pytest.approx(rp["achieved"] / 1000.0)
    assert rp["traffic"] == pytest.approx(bench.DRAM_PER_UNIT["k_prefix"] * n)
    # the headline is the step's largest kernel that has a formula
    assert r["roofline"]["kernel"] == "k_prefix"
    bd = r["rooflines"]["k_bucket_direct"]
    assert bd["algo_bytes"] == 24 * n and bd["kernel_ms"] == pytest.approx(0.002)
    st = r["rooflines"]["sort_stage"]
    assert st["algo_bytes"] == 72 * n + 20 * n
