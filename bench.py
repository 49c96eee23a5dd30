"""Benchmark of the prefix-doubling string sort (one JSON line on stdout).

Default workload (N=1): 32,000,000 strings of 200 bytes over 'A'-'Z', D/N 0.25
(44 'A's + 6 base-26 digits of a seeded permutation + 150 random letters),
split into p = 64 contiguous equal PEs, sorted on one B200 by dsss_pd_sort.

  value     strings/s with the input resident in HBM (device-timed, max over ranks)
  e2e       the same metric through dsss_pd_sort_host: pinned host input copied
            in, results copied out, inside the timed region
  roofline  the dominant kernel of one sort against HBM: algorithmic bytes
            per launch over its CUDA-event launch time (the formulas are
            listed in ROOFLINE_BYTES); traffic = DRAM bytes per unit from one
            ncu capture on 8e6 strings times the units of one launch (a
            capture of the full launch is beyond the capture-size rule)
  rooflines the same figure for every kernel with a formula, and for the
            string sort stage (D + 20 n, D = sum of DP lengths: 8 B id read +
            8 B id write + 4 B LCP write per string) and for the sort plus
            merge stages (D + 20 n + sum(DP - lcp + 1) + 24 n)
  dn100m    the same sort of 1e8 strings x 100 B (D/N 0.5, p = 64),
            generated on the device, with its own rooflines
  ms_path   the merge-sort path (dsss_ms_sort) on the same input, device-timed
  hq_path   hQuicksort (dsss_hq_sort, the reference's RQuick competitor) on
            the same input, device-timed
  formats   the input side (dsss_distribute_lines on a 1.6 GB text) and the
            varint LCP coding (32e6 values), device-timed
  cpu_baseline  the oracle port of the reference path on the host

--mode ms / --mode hq time the merge-sort path or hQuicksort alone (one GPU).
--impl reference times the reference's own prefix_doubling executable
(compiled from its sources into oracle/_ref over a process-based MPI stand-in)
on the same input with p ranks on the host cores: the median of its
`sorting_overall` times (run_reference).
Under torchrun (N > 1) the default is --mode dist: one distributed sort over
all ranks, each rank holding p PEs of its own 32e6-string share (weak
scaling), with the hash exchange of every round, the sample all-gather and
the string all-to-all over NCCL; --mode replicas runs one independent sort
per GPU instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (n, len, k, p, description, further generator arguments)
    "dn32m": (32_000_000, 200, 50, 64, "32e6 strings x 200 B, D/N 0.25, p = 64 PEs", {}),
    "dn1m": (1_000_000, 100, 50, 4, "1e6 strings x 100 B, D/N 0.5, p = 4 PEs", {}),
    "dn8m": (8_000_000, 200, 50, 64, "8e6 strings x 200 B, D/N 0.25, p = 64 PEs (profiling size)", {}),
    "dn100m": (100_000_000, 100, 50, 64, "1e8 strings x 100 B, D/N 0.5, p = 64 PEs", {}),
    "skew20m": (20_000_000, 100, 20, 64, "20e6 strings, 80 % x 100 B with k = 20 and 20 % x 500 B with k = 400 "
                "(seeded choice), p = 64 PEs", dict(long_len=500, long_k=400, frac_long=0.2)),
}


# DRAM bytes (read + write) per unit of the kernels that carry a roofline,
# from one ncu capture each on 8e6 strings x 200 B (D/N 0.25, p = 64); the
# traffic of a launch grows with its units.  None: not captured.
DRAM_PER_UNIT = {"k_prefix": 234.6, "k_pp_hist1": None, "k_pp_scatter1": 13.5, "k_pp_hist2": None,
                 "k_pp_scatter2": 18.8, "k_dp_bucket_dups": 8.1, "k_dp_lens": None, "k_bucket_direct": 18.1,
                 "k_ms_scatter_pay": 18.2}


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1].split()[0]))
                mx.append(float(c[2].split()[0]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_port(n_sample, L, k, p, seed, gk=None):
    """Oracle port, one thread, on a bounded sample of the workload."""
    import __graft_entry__
    import oracle
    d = __graft_entry__.load_package()
    hs = d.gen_dn(n_sample, L, k, seed=seed, **(gk or {}))
    s = oracle.Strings.from_host(hs)
    t = time.perf_counter()
    oracle.pd_sort(s, d.equal_parts(hs.n, p))
    return hs.n / (time.perf_counter() - t)


def uneven_sizes(nsets, lo, hi, seed):
    """Seeded log-uniform sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return [int(x) for x in np.exp(rng.uniform(np.log(lo), np.log(hi), size=nsets))]


def bench_batched(d, torch, steps, warmup, p=64, nsets=16, text=4 << 20, sizes=None):
    """Suffix instances (all suffixes, truncated to 256 B, of seeded order-3
    Markov ACGT texts with 1% copied 1-4 KiB blocks): nsets texts of `text`
    bytes (or of the given uneven sizes) sorted as one dsss_pd_sort_batched
    call vs one dsss_pd_sort call per instance, inputs resident in HBM,
    device-timed."""
    texts = sizes if sizes is not None else [text] * nsets
    nsets = len(texts)
    sets = [d.gen_suffix_strings(t, 256, seed=100 + k) for k, t in enumerate(texts)]
    hs, sb = d.concat_sets(sets)
    pb = d.batched_parts(sb, p)
    ds_all = d.DeviceStrings(hs)
    ds_each = [d.DeviceStrings(h) for h in sets]
    ctx = d.Context(torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    n = hs.n
    out, outs = None, [None] * nsets

    def batched():
        nonlocal out
        out = d.pd_sort_batched(ctx, ds_all, nsets, p, pb, out=out)

    def plain():
        for k in range(nsets):
            outs[k] = d.pd_sort(ctx, ds_each[k], p, out=outs[k])

    tuning = d.autotune(ctx, ds_all, p, part_begin=pb, nsets=nsets, trials=2)
    res = {}
    for name, fn in (("plain", plain), ("batched", batched)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / steps
    # the batched result equals the per-instance results
    same = all(np.array_equal(out["dp"][int(sb[k]):int(sb[k + 1])].cpu().numpy(),
                              outs[k]["dp"][:sets[k].n].cpu().numpy()) for k in range(nsets))
    char_bytes = int(hs.lengths.astype(np.uint64).sum()) + n
    ctx.close()
    desc = (f"{nsets} x {text >> 20} MiB-text suffix instances (x 256 B max), p = {p} each" if sizes is None else
            f"{nsets} suffix instances (x 256 B max) of uneven texts, log-uniform {min(texts)}..{max(texts)} bytes "
            f"(seed 77), p = {p} each")
    return {
        "workload": desc, "text_bytes": texts,
        "strings": n, "char_bytes": char_bytes, "steps": steps,
        "plain_ms": res["plain"], "batched_ms": res["batched"],
        "plain_strings_per_s": n / (res["plain"] * 1e-3), "batched_strings_per_s": n / (res["batched"] * 1e-3),
        "batched_char_gbs": char_bytes / (res["batched"] * 1e-3) / 1e9,
        "speedup": res["plain"] / res["batched"], "dp_identical": bool(same), "tuning": tuning,
    }


def bench_serving(d, torch, p=8, n_req=48, rate=250.0, seed=2024, workers=6, max_batch=2_000_000,
                  reserve=24 << 30):
    """Sort requests through dsss_server: n log-uniform in [1e3, 4e6], lengths
    Zipf(1.2) on [8, 256], bytes 0x21-0x7E after a shared random prefix; host
    buffers pinned.  Saturated throughput (all requests queued at once) and
    latency under seeded Poisson arrivals at `rate` requests/s, for continuous
    batching (`workers` batches in flight, up to `max_batch` strings per batch
    beyond its first request) and for the plain per-request path (1 worker,
    one request per batch = dsss_pd_sort_host per request).  Both servers map
    `reserve` bytes into their memory pool at start; admission is against a
    150 GB budget."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(4e6), size=n_req)).astype(np.int64)
    reqs = [d.gen_request(int(n), seed=seed * 1000 + k, pinned=True) for k, n in enumerate(ns)]
    gaps = rng.exponential(1.0 / rate, size=n_req)
    arrivals = np.cumsum(gaps) - gaps[0]
    total = int(ns.sum())
    outs = []
    for h in reqs:
        mk = (lambda: d._alloc_host(max(h.n, 1) * 4, np.uint32, True)[:max(h.n, 1)])
        outs.append(dict(local_order=mk(), dp=mk(), perm_index=mk(), perm_pe=mk(), merged_lcp=mk(),
                         intervals=np.zeros(p * p, np.uint64), recv_counts=np.zeros(p, np.uint64)))

    def run(workers, max_sets, paced, mbs=0):
        srv = d.Server(torch.cuda.current_device(), p=p, workers=workers, max_sets=max_sets, max_batch_strings=mbs,
                       reserve_bytes=reserve, hbm_budget=150_000_000_000)
        for h, o in list(zip(reqs, outs))[:4]:  # warm-up
            srv.wait(srv.submit(h, out=o)[0])
        t0 = d.clock_now()
        tickets = []
        for k, (h, o) in enumerate(zip(reqs, outs)):
            if paced:
                dt = t0 + arrivals[k] - d.clock_now()
                if dt > 0:
                    time.sleep(dt)
            tickets.append(srv.submit(h, out=o)[0])
        st = [srv.wait(t) for t in tickets]
        info = srv.info()
        srv.close()
        lat = np.array([s["latency"] for s in st]) * 1e3
        span = max(s["t_done"] for s in st) - min(s["t_submit"] for s in st)
        return {"strings_per_s": total / span, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_batch": info["batched_requests"] / info["batches"],
                "max_reserved_gb": info["max_reserved_bytes"] / 1e9}

    served_sat = run(workers, 0, False, max_batch)
    plain_sat = run(1, 1, False)
    served = run(workers, 0, True, max_batch)
    plain = run(1, 1, True)
    return {
        "workload": f"{n_req} requests, n log-uniform [1e3, 4e6] (total {total}), p = {p}, Poisson {rate}/s (seed {seed})",
        "hbm_budget_gb": 150, "workers": workers, "max_batch_strings": max_batch,
        "served": {"saturated_strings_per_s": served_sat["strings_per_s"], "p50_ms": served["p50_ms"],
                   "p99_ms": served["p99_ms"], "paced_strings_per_s": served["strings_per_s"],
                   "mean_batch": served_sat["mean_batch"], "max_reserved_gb": served_sat["max_reserved_gb"]},
        "plain": {"saturated_strings_per_s": plain_sat["strings_per_s"], "p50_ms": plain["p50_ms"],
                  "p99_ms": plain["p99_ms"], "paced_strings_per_s": plain["strings_per_s"]},
        "speedup_saturated": served_sat["strings_per_s"] / plain_sat["strings_per_s"],
    }


def bench_formats(d, torch, steps):
    """The input side and the LCP wire format on one GPU, device-timed:
    dsss_distribute_lines on a 1.6 GB text in pinned host memory (8e6 lines of
    the D/N rule, 200 B, p = 64, the line bound given; the call takes host
    bytes, so its time includes the host-to-device copy of the text, and the
    kernels alone are timed as well), and varint
    coding of 32e6 LCP-like values (uniform 0..199, every 64th up to 2^20) over
    64 destination ranges."""
    hs = d.gen_dn(8_000_000, 200, 50, seed=7)
    lines = hs.n
    pinned = torch.empty(hs.char_bytes, dtype=torch.uint8, pin_memory=True)
    text = pinned.numpy()
    text[:] = hs.chars[:hs.char_bytes]
    del hs
    text[text == 0] = 10
    ctx = d.Context(0)
    stream = torch.cuda.current_stream()
    out = {}
    for _ in range(2):
        ds, pb = d.distribute_lines(ctx, text, 64, cap_n=lines + 1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ds, pb = d.distribute_lines(ctx, text, 64, cap_n=lines + 1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ctx.set_timing(True)
    ds, pb = d.distribute_lines(ctx, text, 64, cap_n=lines + 1)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    kms = sum(v[1] for k2, v in kt.items() if k2.startswith("k_lines") or k2.startswith("scan"))
    out["distribute_lines"] = {"bytes": int(text.size), "lines": ds.n, "ms_per_call": ms,
                               "gbs_e2e": text.size / (ms * 1e-3) / 1e9, "kernels_ms": round(kms, 4),
                               "gbs_kernels": text.size / (kms * 1e-3) / 1e9}
    del ds, text, pinned
    n = 32_000_000
    g = torch.Generator(device="cuda").manual_seed(11)
    vals = torch.randint(0, 200, (n,), device="cuda", dtype=torch.int32, generator=g)
    vals[::64] = torch.randint(0, 1 << 20, (n // 64,), device="cuda", dtype=torch.int32, generator=g)
    rc = np.full(64, n // 64, np.uint64)
    for _ in range(2):
        enc, per = d.varint_encode(ctx, vals, rc)
        dec = d.varint_decode(ctx, enc, n)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        enc, per = d.varint_encode(ctx, vals, rc)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1) / steps
    e0.record(stream)
    for _ in range(steps):
        dec = d.varint_decode(ctx, enc, n)
    e1.record(stream)
    torch.cuda.synchronize()
    dms = e0.elapsed_time(e1) / steps
    assert bool((dec.to(torch.int64) == vals.to(torch.int64)).all())
    out["varint"] = {"values": n, "coded_bytes": int(enc.numel()), "encode_ms": ems, "decode_ms": dms,
                     "encode_values_per_s": n / (ems * 1e-3), "decode_values_per_s": n / (dms * 1e-3)}
    ctx.close()
    return out


def run_dist(args, cfg):
    """--mode dist: one distributed sort over all ranks (dist.py), each rank
    holding p PEs of n strings of the D/N rule (rank-seeded), exchanging over
    NCCL; device-timed per step, max over ranks."""
    import datetime
    import torch
    import torch.distributed as tdist
    import __graft_entry__
    d = __graft_entry__.load_package()
    import dsss_b200.dist as D
    n, L, k, p, desc, gk = cfg
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world == 1:
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        tdist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                 timeout=datetime.timedelta(seconds=300))
    else:
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ctx = d.Context(local)
    be = D.GpuBackend(ctx)
    ds = d.gen_dn_device(ctx, n, L, k, seed=1 + rank, **gk)  # each rank's share, made on its GPU
    pb = d.equal_parts(n, p).astype(np.int64)
    comm = D.Comm()
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        res = D.sort(comm, be, ds, pb)
    phases = {}
    D.sort(comm, be, ds, pb, phases=phases)  # one call with per-phase wall-clock times
    tdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            res = D.sort(comm, be, ds, pb)
        e1.record(stream)
        torch.cuda.synchronize()
    tdist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], device=f"cuda:{local}")
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    ms = float(t.item())
    clocks = clk.summary()
    # the library's kernel launches of one step (CUDA-event timing on)
    ctx.set_timing(True)
    D.sort(comm, be, ds, pb)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    launches = sum(v[0] for k2, v in kt.items() if not k2.startswith("stage:"))
    # end to end: each step copies the rank's strings in from pinned host
    # memory and its merged permutation and LCPs out
    hchars = ds.chars.cpu().pin_memory()
    hoffs = ds.offsets.cpu().pin_memory()
    hlens = ds.lengths.cpu().pin_memory()
    dchars, doffs, dlens = torch.empty_like(ds.chars), torch.empty_like(ds.offsets), torch.empty_like(ds.lengths)
    dse = d.DeviceStrings(None, chars=dchars, offsets=doffs, lengths=dlens, char_bytes=ds.char_bytes)
    outs = [torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(3)]

    def e2e_step():
        dchars.copy_(hchars, non_blocking=True)
        doffs.copy_(hoffs, non_blocking=True)
        dlens.copy_(hlens, non_blocking=True)
        r = D.sort(comm, be, dse, pb)
        m = int(r.get("recv_total", 0))
        for o, key in zip(outs, ("perm_index", "perm_pe", "merged_lcp")):
            if m:
                o[:m].copy_(r[key][:m], non_blocking=True)
        return m

    e2e_step()
    tdist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    recv = 0
    for _ in range(args.steps):
        recv = e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    tdist.barrier()
    ems = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ems], device=f"cuda:{local}")
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    ems = float(t.item())
    # one rank: the staged path too (local sort, DP rounds with their
    # exchanges, partition, bucket send, all-to-all, regroup, merge), with the
    # receive containers merged by one sort and by co-ranked tiles
    staged = None
    if world == 1:
        staged = {}
        for mode in (1, 2):
            with d.tuned(merge_by_sort=mode):
                D.sort(comm, be, ds, pb, fused=False)
                torch.cuda.synchronize()
                ph2 = {}
                t0 = time.perf_counter()
                D.sort(comm, be, ds, pb, fused=False, phases=ph2)
                torch.cuda.synchronize()
                wall = (time.perf_counter() - t0) * 1e3
                ctx.set_timing(True)
                D.sort(comm, be, ds, pb, fused=False)
                torch.cuda.synchronize()
                kt2 = ctx.kernel_times()
                ctx.set_timing(False)
                top = sorted(((k2, v[1]) for k2, v in kt2.items() if not k2.startswith("stage:")), key=lambda x: -x[1])
                staged[f"merge_by_sort={mode}"] = {"ms_per_call": wall,
                                                   "phases_ms": {k: round(v, 3) for k, v in ph2.items()},
                                                   "kernels_ms": {k2: round(v, 3) for k2, v in top[:16]}}
    if rank == 0:
        line = {
            "metric": "strings/s", "value": n * world / (ms * 1e-3), "unit": "strings/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded D/N generator)",
            "config": {"workload": desc + f", {world} GPU(s) x {p} PEs, one distributed sort", "n_per_gpu": n,
                       "len": L, "p_per_gpu": p, "parallelism": f"{world} ranks, NCCL exchanges (dist.py)",
                       "l2": "inputs > L2, no flush"},
            "mode": "dist", "dp_rounds": res.get("dp_rounds"), "clocks": clocks,
            "gpu_launches": int(launches * args.steps),
            "e2e": {"value": n * world / (ems * 1e-3), "unit": "strings/s",
                    "h2d_bytes_per_step": int(ds.char_bytes + d.PAD + 12 * n), "d2h_bytes_per_step": 12 * recv,
                    "ms_per_step": ems},
            "phases_ms": {k: round(v, 3) for k, v in phases.items()},
            "staged_one_rank": staged,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    tdist.destroy_process_group()


def config_of(cfg):
    """The line's `config`: identical on the GPU arm and the reference arm."""
    n, L, k, p, desc, gk = cfg
    return {"workload": desc, "n": n, "len": L, "k": k, "p": p, "generator": dict(gk) or None, "seed": 1,
            "l2": "inputs larger than L2 (126 MB), no flush"}


def run_reference(args, cfg):
    """--impl reference: the reference's own prefix_doubling executable
    (src/executables/prefix_doubling.cpp with its default policies, compiled
    from the reference's sources into oracle/_ref over the process-based MPI
    stand-in oracle/shim_mpi) sorting the same input as the GPU arm with p
    ranks = the configuration's p PEs on the host cores.  The input is made by
    the oracle's restatement of the generator (no product code is loaded),
    written one string per line and read by the executable's FileDistributer
    (--generator 2 --path <file> --strongScaling).  One iteration of the
    executable is one step; its time is the `sorting_overall` RESULT (the
    slowest rank); W warm-up iterations are dropped and value = n / median of
    the K timed ones."""
    import shutil
    import oracle
    n, L, k, p, desc, gk = cfg
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    if not oracle.ref_exe_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/prefix_doubling was not built (the "
                          "reference tree was absent when oracle/ was built)"}), flush=True)
        return
    s = oracle.gen_dn(n, L, k, seed=1, **gk)
    tmpdir = "/dev/shm" if os.path.isdir("/dev/shm") and shutil.disk_usage("/dev/shm").free > 3 * s.char_bytes \
        else tempfile.gettempdir()
    path = os.path.join(tmpdir, f"dsss_ref_input_{os.getpid()}.txt")
    try:
        oracle.write_lines(s, path)
        char_bytes = int(s.char_bytes)
        del s
        iters = args.warmup + args.steps
        times, _ = oracle.run_reference_pd(path, p, iters)
    finally:
        if os.path.exists(path):
            os.unlink(path)
    if len(times) != iters:
        raise RuntimeError(f"expected {iters} iterations, parsed {len(times)}")
    timed = times[args.warmup:]
    sec = statistics.median(timed)
    value = n / sec
    line = {
        "impl": "reference", "metric": "strings/s", "value": value, "unit": "strings/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded D/N generator)",
        "config": config_of(cfg),
        "char_gbs": char_bytes / sec / 1e9,
        "cpu_baseline": {"value": value, "unit": "strings/s", "cores": cores, "kind": "reference",
                         "sample": f"the whole input ({n} strings, {char_bytes} bytes): the reference's "
                                   f"prefix_doubling with {p} ranks (processes) on {cores} host cores, "
                                   f"default policies, median sorting_overall of {args.steps} iterations after "
                                   f"{args.warmup}"},
        "e2e": {"value": value, "unit": "strings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iteration_ms": [round(t * 1e3, 2) for t in times],
    }
    print(json.dumps(line), flush=True)


def run_path(args, cfg, which):
    """--mode ms / hq: the merge-sort path (dsss_ms_sort) or hQuicksort
    (dsss_hq_sort) alone on the same input, one GPU, device-timed, with its
    stage and kernel times."""
    import torch
    import __graft_entry__
    d = __graft_entry__.load_package()
    n, L, k, p, desc, gk = cfg
    hs = d.gen_dn(n, L, k, seed=1, **gk)
    ds = d.DeviceStrings(hs)
    del hs
    ctx = d.Context(0)
    fn = d.ms_sort if which == "ms" else d.hq_sort
    stream = torch.cuda.current_stream()
    out = None
    for _ in range(args.warmup):
        out = None
        out = fn(ctx, ds, p)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            out = None
            out = fn(ctx, ds, p)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ctx.set_timing(True)
    out = None
    out = fn(ctx, ds, p)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    name = {"ms": "merge-sort path (dsss_ms_sort: whole strings and LCPs per receiving PE)",
            "hq": "hQuicksort (dsss_hq_sort: RQuick, seed 3469931 + rank; whole strings per PE)"}[which]
    line = {
        "metric": "strings/s", "value": n / (ms * 1e-3), "unit": "strings/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded D/N generator)", "mode": which,
        "config": {"workload": desc + ", " + name, "n": n, "len": L, "p": p,
                   "l2": "inputs > L2 (126 MB), no flush"},
        "out_char_bytes": out["char_bytes"], "clocks": clk.summary(),
        "stages_ms": {k2[6:]: round(v[1], 4) for k2, v in kt.items() if k2.startswith("stage:")},
        "kernels_ms": {k2: round(v[1], 4) for k2, v in sorted(kt.items(), key=lambda x: -x[1][1])
                       if not k2.startswith("stage:")},
    }
    print(json.dumps(line), flush=True)


# Algorithmic bytes of the kernels that carry a roofline, per step of one
# sort (n strings, lengths L, DP lengths dp, schedule depths 8, 24, 40, 72, ...):
#   k_prefix   the string sort's first pass over the arena: each string's
#              first min(L + 1, 72) bytes read once, its 8-byte key and the
#              four 8-byte prefix hashes of the dense rounds written, its id
#              and handle read (16 + 4 B): min(L + 1, 72) + 60 per string
#   k_dp_part  the dense hash round's partition: for every string hashed at
#              its final depth, the stored 8-byte hash read and the 12-byte
#              (hash, string) pair written: 20 per string
#   k_dp_bucket_dups  the pairs read back: 12 per string
#   k_dp_lens  per sorted position the 4-byte id read, the 16-byte handle
#              gathered and 12 bytes written: 32 per string
ROOFLINE_BYTES = {
    "k_prefix": "sum over strings of (min(L + 1, 72) + 36)",
    "k_pp_hist1": "8 per string hashed at its final depth",
    "k_pp_scatter1": "20 per string hashed at its final depth",
    "k_pp_hist2": "8 per string hashed at its final depth",
    "k_pp_scatter2": "24 per string hashed at its final depth",
    "k_dp_bucket_dups": "12 per string hashed at its final depth",
    "k_dp_lens": "32 per string",
    "k_bucket_direct": "24 per string",
    "k_ms_scatter_pay": "24 per string (the multisplit by PE)",
}
SORT_KERNELS = ("k_init", "k_tile_counts", "k_prefix", "k_keys_diff", "k_hist", "k_chunk_sum", "k_seg_scan",
                "k_scatter", "k_seg_sort", "k_warp_segs", "k_spec", "k_pivot", "k_seg_offsets", "k_split_sample",
                "k_lcp_fix", "scan_")


def pd_rooflines(out, lengths, n, kt, steps, peak, peak_kind, traffic_known=True):
    """Rooflines of one dsss_pd_sort step from its per-kernel event times."""
    kernels = {k: v for k, v in kt.items() if not k.startswith("stage:")}
    stages = {k[6:]: v[1] / steps for k, v in kt.items() if k.startswith("stage:")}
    dp = out["dp"][:n].cpu().numpy().view(np.uint32).astype(np.uint64)
    lcp = out["merged_lcp"][:n].cpu().numpy().view(np.uint32).astype(np.uint64)
    L = np.asarray(lengths, np.uint64)
    D = int(dp.sum())
    sched = np.array([8] + [8 + (16 << j) for j in range(26)], np.uint64)
    hashed = int(np.isin(dp, sched).sum())
    per_step = {
        "k_prefix": int(np.minimum(L + 1, 72).sum()) + 36 * n,
        "k_pp_hist1": 8 * hashed,
        "k_pp_scatter1": 20 * hashed,
        "k_pp_hist2": 8 * hashed,
        "k_pp_scatter2": 24 * hashed,
        "k_dp_bucket_dups": 12 * hashed,
        "k_dp_lens": 32 * n,
        "k_bucket_direct": 24 * n,
        "k_ms_scatter_pay": 24 * n,
    }
    b_sort = D + 20 * n
    b_merge = int((dp - np.minimum(lcp, dp) + 1).sum()) + 24 * n
    sort_ms = sum(v[1] for k, v in kernels.items() if k.startswith(SORT_KERNELS)) / steps
    sort_launches = sum(v[0] for k, v in kernels.items() if k.startswith(SORT_KERNELS)) / steps

    def line(kernel, algo, ms, launches, formula, traffic=None, note=None):
        ach = algo / (ms * 1e-3) / 1e9 if ms > 0 else float("nan")
        r = {"bound": "hbm", "kernel": kernel, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
             "peak_kind": peak_kind, "traffic": traffic, "algo_bytes": algo, "algo_formula": formula,
             "kernel_ms": ms, "launches": launches}
        if note:
            r["traffic_note"] = note
        return r

    per = {}
    for k, formula in ROOFLINE_BYTES.items():
        if k not in kernels:
            continue
        launches = kernels[k][0] / steps
        ms = kernels[k][1] / steps
        unit = DRAM_PER_UNIT.get(k)
        units = n if k in ("k_prefix", "k_dp_lens", "k_bucket_direct", "k_ms_scatter_pay") else hashed
        traffic = unit * units if (unit and traffic_known) else None
        # the step's bytes over the step's time of the kernel (all its launches)
        per[k] = line(k, per_step[k], ms, launches, formula + " (per step: all launches)", traffic,
                      "ncu DRAM bytes per string on 8e6 strings x 200 B (D/N 0.25), times the strings"
                      if traffic is not None else "not captured for this string mix")
    ranked = sorted(kernels.items(), key=lambda kv: -kv[1][1])
    top = ranked[0][0] if ranked else None
    rl = {
        "sort_stage": line("string sort K3 (all launches of the sort stage)", b_sort, sort_ms, sort_launches,
                           "D + 20 n"),
        "sort_merge": line("sort + merge stages (north-star target)", b_sort + b_merge,
                           stages.get("sort", 0.0) + stages.get("merge", 0.0), None,
                           "D + 20 n + sum(DP - lcp + 1) + 24 n"),
    }
    rl.update(per)
    # the headline: the step's largest kernel among those with a formula
    main = next((per[k] for k, _ in ranked if k in per), rl["sort_stage"])
    return {"roofline": dict(main, top_kernel=top), "rooflines": rl, "stages_ms": stages,
            "kernels_ms": {k: round(v[1] / steps, 4) for k, v in ranked},
            "launches_per_step": sum(v[0] for v in kernels.values()) / steps}


def bench_config_device(d, torch, name, steps, warmup, peak, peak_kind):
    """One configuration's dsss_pd_sort with its input generated on the
    device (dsss_gen_dn_dev), device-timed, with its stage and kernel times
    and rooflines."""
    n, L, k, p, desc, gk = CONFIGS[name]
    ctx = d.Context(torch.cuda.current_device())
    ds = d.gen_dn_device(ctx, n, L, k, seed=1, **gk)
    stream = torch.cuda.current_stream()
    out = None
    for _ in range(warmup):
        out = d.pd_sort(ctx, ds, p, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        out = d.pd_sort(ctx, ds, p, out=out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ctx.set_timing(True)
    for _ in range(steps):
        out = d.pd_sort(ctx, ds, p, out=out)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    lengths = ds.lengths.cpu().numpy().view(np.uint32)
    roof = pd_rooflines(out, lengths, n, kt, steps, peak, peak_kind, traffic_known=False)
    res = {"workload": desc + " (generated on the device)", "n": n, "len": L, "p": p, "steps": steps,
           "ms_per_step": ms, "strings_per_s": n / (ms * 1e-3),
           "char_gbs": (int(lengths.astype(np.uint64).sum()) + n) / (ms * 1e-3) / 1e9,
           "roofline": roof["roofline"], "rooflines": roof["rooflines"], "stages_ms": roof["stages_ms"],
           "kernels_ms": dict(list(roof["kernels_ms"].items())[:16])}
    del out, ds
    ctx.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="dn32m", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-ms", action="store_true", help="skip the merge-sort path line")
    ap.add_argument("--no-hq", action="store_true", help="skip the hQuicksort line")
    ap.add_argument("--no-formats", action="store_true", help="skip the line distribution and varint lines")
    ap.add_argument("--no-dn100m", action="store_true", help="skip the 1e8-string configuration")
    ap.add_argument("--no-autotune", action="store_true", help="skip dsss_autotune before the warm-up")
    ap.add_argument("--mode", default=None, choices=["replicas", "dist", "ms", "hq"],
                    help="replicas: one independent sort per GPU (the default on one GPU); dist: one sort over "
                         "all GPUs with the exchanges over NCCL (the default on several GPUs); ms / hq: the "
                         "merge-sort path or hQuicksort alone on one GPU")
    ap.add_argument("--tune", action="append", default=[], metavar="KNOB=VALUE",
                    help="set a tuning knob (dsss_tune_set) before the run; repeatable")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    cfg = CONFIGS[args.config]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.mode is None:
        args.mode = "dist" if world > 1 else "replicas"

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, cfg)
        return
    if args.mode == "dist":
        run_dist(args, cfg)
        return
    if args.mode in ("ms", "hq"):
        if rank == 0:
            run_path(args, cfg, args.mode)
        return

    import torch
    import __graft_entry__
    d = __graft_entry__.load_package()
    for kv in args.tune:
        name, value = kv.split("=", 1)
        d.tune_set(name, int(value))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    n, L, k, p, desc, gk = cfg
    hs = d.gen_dn(n, L, k, seed=1 + rank, pinned=not args.no_e2e, **gk)
    ds = d.DeviceStrings(hs, f"cuda:{local}")
    ctx = d.Context(local)
    stream = torch.cuda.current_stream()
    out = None

    def barrier():
        if dist is not None:
            dist.barrier()

    # knobs picked by the autotuner on this input (results never depend on them)
    tuning = None if args.no_autotune else d.autotune(ctx, ds, p, trials=2)
    for _ in range(args.warmup):
        out = d.pd_sort(ctx, ds, p, out=out)
    torch.cuda.synchronize()

    # timed region: K steps, device events on the launching stream
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            out = d.pd_sort(ctx, ds, p, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.summary()

    # per-kernel events (a second pass of the same K steps with timing on)
    ctx.set_timing(True)
    for _ in range(args.steps):
        out = d.pd_sort(ctx, ds, p, out=out)
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    peak, peak_kind = read_peaks()
    roof = pd_rooflines(out, hs.lengths, n, kt, args.steps, peak, peak_kind, traffic_known=not gk)
    char_bytes = int(hs.lengths.astype(np.uint64).sum()) + n
    value = n * world / (ms * 1e-3)

    # the 1e8-string configuration (generated on the device), one GPU
    dn100m = None
    if world == 1 and not args.no_dn100m and args.config != "dn100m":
        del out
        out = None
        torch.cuda.empty_cache()
        dn100m = bench_config_device(d, torch, "dn100m", max(3, min(args.steps, 10)), 3, peak, peak_kind)
        torch.cuda.empty_cache()

    # e2e through the host entry point
    e2e = None
    if not args.no_e2e:
        hout = None
        for _ in range(1):
            hout = d.pd_sort_host(ctx, hs, p, out=hout, pinned=True)
        barrier()
        torch.cuda.synchronize()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(args.steps):
            hout = d.pd_sort_host(ctx, hs, p, out=hout, pinned=True)
        h1.record(stream)
        torch.cuda.synchronize()
        ems = h0.elapsed_time(h1) / args.steps
        if dist is not None:
            t = torch.tensor([ems], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        h2d = hs.char_bytes + d.PAD + n * 12
        d2h = n * 4 * 5 + p * p * 8
        e2e = {"value": n * world / (ems * 1e-3), "unit": "strings/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = min(n, 8_000_000)
        cpu = {"value": cpu_baseline_port(sample, L, k, p, seed=1, gk=gk), "unit": "strings/s", "cores": 1, "kind": "port",
               "sample": f"{sample} strings of the same rule, p = {p}, oracle port single-threaded"}

    # the merge-sort path (dsss_ms_sort) on the same input, device-timed
    ms_path = None
    if world == 1 and not args.no_ms:
        del out
        torch.cuda.empty_cache()
        mout = None
        for _ in range(2):
            mout = d.ms_sort(ctx, ds, p)
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        msteps = max(3, min(args.steps, 10))
        for _ in range(msteps):
            mout = d.ms_sort(ctx, ds, p)
        m1.record(stream)
        torch.cuda.synchronize()
        mms = m0.elapsed_time(m1) / msteps
        ms_path = {"workload": desc + ", merge-sort path (whole strings and LCPs per receiving PE)",
                   "steps": msteps, "ms_per_call": mms, "strings_per_s": n / (mms * 1e-3),
                   "out_char_bytes": mout["char_bytes"], "avg_lcp": mout["avg_lcp"]}
        del mout
        out = None

    # hQuicksort (dsss_hq_sort) on the same input, device-timed
    hq_path = None
    if world == 1 and not args.no_hq:
        out = None
        torch.cuda.empty_cache()
        hout = None
        for _ in range(2):
            hout = d.hq_sort(ctx, ds, p)
        torch.cuda.synchronize()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        hsteps = max(3, min(args.steps, 10))
        for _ in range(hsteps):
            hout = d.hq_sort(ctx, ds, p)
        h1.record(stream)
        torch.cuda.synchronize()
        hms = h0.elapsed_time(h1) / hsteps
        cnt = np.asarray(hout["counts"], np.int64)
        ctx.set_timing(True)
        for _ in range(3):
            hout = d.hq_sort(ctx, ds, p)
        torch.cuda.synchronize()
        hkt = ctx.kernel_times()
        ctx.set_timing(False)
        hq_stages = {k2[6:]: round(v[1] / 3, 4) for k2, v in hkt.items() if k2.startswith("stage:")}
        hq_kernels = {k2: round(v[1] / 3, 4) for k2, v in sorted(hkt.items(), key=lambda x: -x[1][1])
                      if not k2.startswith("stage:")}
        hq_path = {"workload": desc + ", hQuicksort (RQuick, seed 3469931 + rank; whole strings per PE)",
                   "steps": hsteps, "ms_per_call": hms, "strings_per_s": n / (hms * 1e-3),
                   "levels": hout["levels"], "out_char_bytes": hout["char_bytes"],
                   "pe_strings_min": int(cnt.min()), "pe_strings_max": int(cnt.max()),
                   "stages_ms": hq_stages, "kernels_ms": dict(list(hq_kernels.items())[:12])}
        del hout

    ctx.close()
    del ds, out
    torch.cuda.empty_cache()
    # batched and served forms: reported on the one-GPU line
    batched = None
    if world == 1 and not args.no_batched:
        batched = bench_batched(d, torch, max(3, min(args.steps, 10)), 3)
        batched["uneven"] = bench_batched(d, torch, max(3, min(args.steps, 10)), 3,
                                          sizes=uneven_sizes(16, 1 << 14, 4 << 20, 77))
    serving = None
    if world == 1 and not args.no_serving:
        serving = bench_serving(d, torch)
    formats = None
    if world == 1 and not args.no_formats:
        formats = bench_formats(d, torch, max(3, min(args.steps, 10)))

    if rank == 0:
        line = {
            "metric": "strings/s", "value": value, "unit": "strings/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded D/N generator)",
            "config": config_of(cfg),
            "char_bytes": char_bytes,
            "parallelism": "one GPU holds all p PEs" if world == 1 else f"{world} ranks, one instance each (weak)",
            "char_gbs": char_bytes / (ms * 1e-3) / 1e9 * world,
            "roofline": roof["roofline"],
            "rooflines": roof["rooflines"],
            "tuning": tuning,
            "stages_ms": roof["stages_ms"],
            "kernels_ms": roof["kernels_ms"],
            "gpu_launches": int(round(roof["launches_per_step"] * args.steps)),
            "dn100m": dn100m,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "ms_path": ms_path,
            "hq_path": hq_path,
            "batched": batched,
            "serving": serving,
            "formats": formats,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
