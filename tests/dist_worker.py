"""Rank body of the distributed-path tests: runs dist.sort on this rank's PEs
and saves its results (spawned by test_dist.py and test_gpu_dist.py)."""
import datetime
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rank_main(rank, world, port, outdir, inputs, backend, pg="gloo"):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as tdist
    import __graft_entry__
    import oracle
    from dist_oracle import HostArena, OracleBackend, pack_list
    d = __graft_entry__.load_package()
    import dsss_b200.dist as D
    strs, pb, splits, sampler = inputs[:4]
    compress = bool(inputs[4]) if len(inputs) > 4 else False
    mode = inputs[5] if len(inputs) > 5 else "pd"
    golomb = bool(inputs[6]) if len(inputs) > 6 else False
    if pg == "nccl":
        import torch
        torch.cuda.set_device(0)
    tdist.init_process_group(pg, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        q0, q1 = splits[rank], splits[rank + 1]
        s0, s1 = int(pb[q0]), int(pb[q1])
        mine = strs[s0:s1]
        pb_local = np.asarray(pb[q0:q1 + 1], np.int64) - s0
        if backend == "oracle":
            be = OracleBackend(oracle)
            chars, offs, lens, nb = pack_list(mine)
            arena = HostArena(chars, offs, lens, nb)
        else:
            import torch
            torch.cuda.set_device(0)
            ctx = d.Context(0)
            be = D.GpuBackend(ctx)
            arena = be.strings(d.from_bytes_list(mine))
        if mode == "ms":
            res = D.merge_sort(D.Comm(), be, arena, pb_local, compress_lcps=compress)
        else:
            res = D.sort(D.Comm(), be, arena, pb_local, sampler, compress_lcps=compress, golomb=golomb)
        out = {"q0": q0, "q1": q1, "s0": s0}
        if mode == "ms":
            nrecv = int(res.get("recv_total", 0))
            ch = res["chars"]
            ch = ch.cpu().numpy() if hasattr(ch, "cpu") else np.asarray(ch)
            out.update(avg_lcp=int(res["avg_lcp"]), out_chars=np.asarray(ch[:int(res["char_bytes"])], np.uint8),
                       out_offsets=be.to_host(res["offsets"], nrecv), out_lengths=be.to_host(res["lengths"], nrecv),
                       out_lcp=be.to_host(res["lcp"], nrecv))
        nrecv = int(res.get("recv_total", 0))
        for k in ("local_order", "dp", "perm_index", "perm_pe", "merged_lcp"):
            if k in res:
                n = s1 - s0 if k in ("local_order", "dp") else nrecv
                out[k] = be.to_host(res[k], n)
        for k in ("intervals", "recv_counts"):
            if k in res:
                out[k] = np.asarray(res[k], np.int64)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), **out)
    finally:
        tdist.destroy_process_group()
