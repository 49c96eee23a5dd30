"""DistributedPrefixDoublingSort::sort with the PEs spread over several GPUs,
one process per GPU (src/sorter/distributed/prefix_doubling.hpp:200-295).

Each rank holds p_local PEs (contiguous global PE ids) as one string arena and
runs the reference's path; its three exchanges go through torch.distributed
(NCCL over NVLink between GPUs; gloo through host memory in CPU tests and
one-GPU runs of several ranks):

  1. distinguishing prefixes, every round: this rank's hashed candidates are
     routed to the rank owning their slice of the hash range (the reference's
     range-partitioned filter, bloomfilter.hpp:529-656), tested for
     duplicates there and the outcome sent back (:662-817); the loop ends when
     no rank has a candidate left (allreduce);
  2. splitters: every rank packs its PEs' samples (truncated to their
     distinguishing prefixes), the sample is gathered on every rank, sorted
     there (ties by global (PE, index), as RQuick's result has them) and every
     rank searches its PEs for the splitters; the interval tables are gathered;
  3. strings: every rank packs one receive container per destination PE
     (bytes [lcp', dp) + NUL, alltoall.hpp:910-1008), the containers travel
     all-to-all, the receiving rank regroups them by receiver and merges them
     with the LCP merge (merging.hpp:66-123).

The compute is the library's CUDA kernels (GpuBackend); the steps between
collectives are plain host logic shared with any backend that has the same
methods.  Results per rank are those of its PEs: local order, distinguishing
prefixes, interval rows, and the merged (index, PE) permutation and LCPs of
its receiving PEs.
"""
import ctypes

import numpy as np

from . import (Arena, DeviceStrings, PAD, _ptr, _stream_ptr, check, lcp_merge, lcp_merge_strings, lib, local_sort_lcp,
               varint_decode, varint_encode)


# ------------------------------------------------------------- collectives --
class Comm:
    """The collectives the path needs, over a torch.distributed process group.
    With NCCL the payload tensors stay on the GPU; with gloo they are staged
    through host memory."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device_ok = dist.get_backend(group) == "nccl"

    def _home(self):
        import torch
        return torch.device("cuda", torch.cuda.current_device()) if self.device_ok else torch.device("cpu")

    def allreduce_sum(self, x: int) -> int:
        import torch
        t = torch.tensor([int(x)], dtype=torch.int64, device=self._home())
        self.dist.all_reduce(t, group=self.group)
        return int(t.item())

    def allgather_np(self, a):
        """Host int64 arrays of any length from every rank, in rank order."""
        import torch
        dev = self._home()
        a = np.ascontiguousarray(a, dtype=np.int64).ravel()
        n = torch.tensor([a.size], dtype=torch.int64, device=dev)
        ns = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(self.world)]
        self.dist.all_gather(ns, n, group=self.group)
        ns = [int(x.item()) for x in ns]
        m = max(ns + [1])
        buf = torch.zeros(m, dtype=torch.int64, device=dev)
        if a.size:
            buf[:a.size] = torch.from_numpy(a).to(dev)
        outs = [torch.zeros(m, dtype=torch.int64, device=dev) for _ in range(self.world)]
        self.dist.all_gather(outs, buf, group=self.group)
        return [o[:k].cpu().numpy() for o, k in zip(outs, ns)]

    def alltoall_counts(self, counts):
        """counts[t] (ints) to rank t; returns the counts every rank sent here."""
        import torch
        t = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=self._home())
        out = torch.zeros(self.world, dtype=torch.int64, device=self._home())
        self.dist.all_to_all_single(out, t, group=self.group)
        return [int(v) for v in out.cpu().tolist()]

    def alltoall_np(self, rows):
        """rows[t]: host int64 array for rank t; returns what every rank sent here."""
        import torch
        sizes = [int(np.asarray(r).size) for r in rows]
        recv_sizes = self.alltoall_counts(sizes)
        flat = (np.concatenate([np.asarray(r, dtype=np.int64).ravel() for r in rows]) if sum(sizes)
                else np.zeros(0, np.int64))
        got = self.alltoallv(flat, sizes, recv_sizes)
        out, k = [], 0
        for m in recv_sizes:
            out.append(got[k:k + m])
            k += m
        return out

    def alltoallv(self, t, send_counts, recv_counts):
        """Elements of t in rank-ordered runs of send_counts to every rank;
        returns what arrives, on t's device (numpy for a numpy input)."""
        import torch
        if isinstance(t, np.ndarray):
            return self.alltoallv(torch.from_numpy(np.ascontiguousarray(t)), send_counts, recv_counts).numpy()
        dev = (t.device if t.is_cuda else self._home()) if self.device_ok else torch.device("cpu")
        src = t.to(dev)
        dt = src.dtype
        if dt == torch.uint64:
            src = src.view(torch.int64)
        out = torch.empty(int(sum(recv_counts)), dtype=src.dtype, device=dev)
        self.dist.all_to_all_single(out, src.contiguous(), [int(c) for c in recv_counts],
                                    [int(c) for c in send_counts], group=self.group)
        if dt == torch.uint64:
            out = out.view(torch.uint64)
        return out.to(t.device)


# ------------------------------------------------------------------- GPU ----
class _DevArena:
    """An arena over device chars with offsets and lengths on the device."""

    def __init__(self, chars, offsets, lengths, char_bytes):
        self.chars, self.offsets, self.lengths = chars, offsets, lengths
        self.char_bytes = int(char_bytes)
        self.n = int(lengths.shape[0])

    def arena(self):
        return Arena(self.chars.data_ptr(), self.char_bytes, self.offsets.data_ptr(), self.lengths.data_ptr(), self.n)


class GpuBackend:
    """The library's kernels on this rank's GPU (torch tensors for storage)."""

    def __init__(self, ctx, stream=None):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.device = torch.device("cuda", ctx.device)
        self.stream = stream

    def _e(self, n, dtype):
        return self.torch.empty(max(int(n), 1), dtype=dtype, device=self.device)

    def _s(self):
        return _stream_ptr(self.stream)

    def strings(self, hs):
        return DeviceStrings(hs, self.device)

    def arena_from(self, chars, offsets, lengths, char_bytes):
        torch = self.torch
        off = torch.from_numpy(np.ascontiguousarray(offsets, np.int64)).to(self.device)
        ln = torch.from_numpy(np.ascontiguousarray(lengths, np.int64).astype(np.int32)).to(self.device)
        return _DevArena(chars, off, ln, char_bytes)

    def local_sort(self, ds, pb):
        order, lcp = local_sort_lcp(self.ctx, ds, len(pb) - 1, part_begin=np.asarray(pb, np.uint64),
                                    stream=self.stream)
        return order, lcp

    def fused_sort(self, ds, pb, sampler):
        """Every PE on this GPU: the one-GPU path (dsss_pd_sort)."""
        from . import pd_sort
        pb = np.asarray(pb, np.uint64)
        p = len(pb) - 1
        out = pd_sort(self.ctx, ds, p, part_begin=pb, sampler=sampler, stream=self.stream)
        return dict(local_order=out["local_order"], dp=out["dp"], intervals=np.asarray(out["intervals"], np.int64)
                    .reshape(p, p), recv_counts=np.asarray(out["recv_counts"], np.int64), perm_index=out["perm_index"],
                    perm_pe=out["perm_pe"], merged_lcp=out["merged_lcp"])

    def new_dp(self, n):
        return self._e(n, self.torch.int32)

    def dp_classify(self, ds, order, lcp, state, depth, dp):
        torch = self.torch
        n = ds.n
        state_out = self._e(n, torch.uint8)
        hpos = self._e(n, torch.int32)
        hval = self._e(n, torch.int64)
        m = ctypes.c_uint64(0)
        check(lib().dsss_dp_classify_hash(self.ctx.h, ctypes.byref(ds.arena()), _ptr(order), _ptr(lcp), _ptr(state),
                                          depth, _ptr(dp), _ptr(state_out), _ptr(hpos), _ptr(hval), ctypes.byref(m),
                                          self._s()))
        k = m.value
        return state_out, hpos[:k], hval[:k]

    def hash_route(self, hval, hpos, nowner):
        torch = self.torch
        m = int(hval.shape[0])
        oh, op = self._e(m, torch.int64), self._e(m, torch.int32)
        counts = np.zeros(nowner, np.uint64)
        check(lib().dsss_hash_route(self.ctx.h, _ptr(hval), _ptr(hpos), m, nowner, _ptr(oh), _ptr(op), _ptr(counts),
                                    self._s()))
        return oh[:m], op[:m], [int(c) for c in counts]

    def hash_sort(self, hval, hpos):
        """The round's hash records in hash order (dsss_hash_sort)."""
        torch = self.torch
        m = int(hval.shape[0])
        oh, op = self._e(m, torch.int64), self._e(m, torch.int32)
        check(lib().dsss_hash_sort(self.ctx.h, _ptr(hval), _ptr(hpos), m, _ptr(oh), _ptr(op), self._s()))
        return oh[:m], op[:m]

    def golomb_param_hashes(self, count, p):
        return int(lib().dsss_golomb_param_hashes(int(count), int(p)))

    def golomb_encode(self, hval, counts, bs):
        from . import golomb_encode
        words, rw = golomb_encode(self.ctx, hval, counts, bs, stream=self.stream)
        return words, [int(x) for x in rw]

    def golomb_decode(self, words):
        from . import golomb_decode
        vals, bc = golomb_decode(self.ctx, words, max_blocks=max(1, int(words.shape[0])), stream=self.stream)
        return vals, [int(x) for x in bc]

    def hash_dups(self, hval):
        m = int(hval.shape[0])
        dup = self._e(m, self.torch.uint8)
        check(lib().dsss_hash_dups(self.ctx.h, _ptr(hval), m, _ptr(dup), self._s()))
        return dup[:m]

    def dp_apply(self, hpos, dup, state):
        c = ctypes.c_uint64(0)
        n = int(state.shape[0])
        check(lib().dsss_dp_apply(self.ctx.h, _ptr(hpos), _ptr(dup), int(hpos.shape[0]), _ptr(state), n,
                                  ctypes.byref(c), self._s()))
        return int(c.value)

    def take(self, t, idx):
        """Host copy of t at the (few) host positions idx."""
        torch = self.torch
        sel = t[torch.from_numpy(np.asarray(idx, np.int64)).to(t.device)].cpu().numpy()
        if sel.dtype == np.int32:
            sel = sel.view(np.uint32)
        return sel.astype(np.int64)

    def pack(self, ds, ids, trunc=None):
        """Strings ids (host) truncated to trunc (host) -> (device chars, host offsets, host lengths, bytes)."""
        torch = self.torch
        m = len(ids)
        if m == 0:
            return (torch.zeros(PAD, dtype=torch.uint8, device=self.device), np.zeros(0, np.int64),
                    np.zeros(0, np.int64), 0)
        d_ids = torch.from_numpy(np.asarray(ids, np.int64).astype(np.int32)).to(self.device)
        d_tr = None if trunc is None else torch.from_numpy(np.asarray(trunc, np.int64).astype(np.int32)).to(self.device)
        offs, lens = self._e(m, torch.int64), self._e(m, torch.int32)
        nb = ctypes.c_uint64(0)
        args = (self.ctx.h, ctypes.byref(ds.arena()), _ptr(d_ids), _ptr(d_tr), m)
        check(lib().dsss_pack_strings(*args, None, 0, _ptr(offs), _ptr(lens), ctypes.byref(nb), self._s()))
        chars = torch.zeros(nb.value + PAD, dtype=torch.uint8, device=self.device)
        check(lib().dsss_pack_strings(*args, _ptr(chars), nb.value + PAD, _ptr(offs), _ptr(lens), ctypes.byref(nb),
                                      self._s()))
        return chars, offs[:m].cpu().numpy(), lens[:m].cpu().numpy().astype(np.int64), int(nb.value)

    def chars_to_host(self, chars, nbytes):
        return chars[:nbytes].cpu().numpy()

    def chars_from_host(self, a):
        torch = self.torch
        out = torch.zeros(a.size + PAD, dtype=torch.uint8, device=self.device)
        if a.size:
            out[:a.size] = torch.from_numpy(np.ascontiguousarray(a, np.uint8)).to(self.device)
        return out

    def sort_arena(self, a):
        order, _ = local_sort_lcp(self.ctx, a, 1, part_begin=np.array([0, a.n], np.uint64), stream=self.stream)
        return order[:a.n].cpu().numpy().view(np.uint32).astype(np.int64)

    def partition_search(self, ds, pb, order, spl, spl_index, p_global, pe_index, indexed):
        p_local = len(pb) - 1
        iv = np.zeros(p_local * p_global, np.uint64)
        si = np.ascontiguousarray(spl_index, np.uint64)
        pi = np.ascontiguousarray(pe_index, np.uint64)
        pbv = np.ascontiguousarray(pb, np.uint64)
        check(lib().dsss_partition_search(self.ctx.h, ctypes.byref(ds.arena()), p_local, _ptr(pbv), _ptr(order),
                                          ctypes.byref(spl.arena()), _ptr(si), p_global, _ptr(pi),
                                          1 if indexed else 0, _ptr(iv), self._s()))
        return iv.reshape(p_local, p_global).astype(np.int64)

    def bucket_send(self, ds, pb, order, lcp, dp, p_global, q_first, iv_local):
        torch = self.torch
        p_local = len(pb) - 1
        n = ds.n
        pbv = np.ascontiguousarray(pb, np.uint64)
        iv = np.ascontiguousarray(iv_local, np.uint64).ravel()
        total = ctypes.c_uint64(0)
        cbeg = np.zeros(p_global + 1, np.uint64)
        counts = np.zeros(p_global * p_local, np.uint64)
        offs = np.zeros(p_global * p_local, np.uint64)
        cstart, slcp = self._e(n, torch.int32), self._e(n, torch.int32)
        args = (self.ctx.h, ctypes.byref(ds.arena()), p_local, _ptr(pbv), _ptr(order), _ptr(lcp), _ptr(dp), p_global,
                q_first, _ptr(iv))
        check(lib().dsss_bucket_send(*args, None, 0, ctypes.byref(total), _ptr(cbeg), None, _ptr(slcp), _ptr(counts),
                                     _ptr(offs), self._s()))
        chars = torch.zeros(total.value + PAD, dtype=torch.uint8, device=self.device)
        check(lib().dsss_bucket_send(*args, _ptr(chars), total.value + PAD, ctypes.byref(total), _ptr(cbeg),
                                     _ptr(cstart), _ptr(slcp), _ptr(counts), _ptr(offs), self._s()))
        return dict(chars=chars[:total.value], char_start=cstart[:n], lcp=slcp[:n],
                    char_begin=cbeg.astype(np.int64), counts=counts.reshape(p_global, p_local).astype(np.int64))

    def regroup(self, blocks, chars, starts, lcps, n, nbytes):
        torch = self.torch
        blk = np.ascontiguousarray(np.asarray(blocks, np.uint64).reshape(-1, 6))
        dchars = torch.zeros(nbytes + PAD, dtype=torch.uint8, device=self.device)
        dstart, dlcp = self._e(n, torch.int32), self._e(n, torch.int32)
        check(lib().dsss_regroup(self.ctx.h, blk.shape[0], _ptr(blk), _ptr(chars), _ptr(dchars), _ptr(starts),
                                 _ptr(dstart), _ptr(lcps), _ptr(dlcp), n, self._s()))
        return dchars, dstart[:n], dlcp[:n]

    def varint_encode(self, values, range_counts):
        return varint_encode(self.ctx, values, range_counts, stream=self.stream)

    def varint_decode(self, data, n):
        return varint_decode(self.ctx, data, n, stream=self.stream)

    def merge(self, chars, nbytes, starts, lcps, counts, offsets):
        out = lcp_merge(self.ctx, chars, nbytes, lcps, counts, offsets, char_start=starts, stream=self.stream)
        return {k: out[k] for k in ("perm_index", "perm_pe", "merged_lcp")}

    def lcp_sum(self, lcp, n):
        return int(lcp[:n].to(self.torch.int64).sum().item()) if n else 0

    def lengths_in_order(self, ds, order):
        """Whole strings as DP: the length of the string at every local position."""
        n = ds.n
        if n == 0:
            return self._e(1, self.torch.int32)
        return ds.lengths[:n][order[:n].to(self.torch.int64) & 0xFFFFFFFF].to(self.torch.int32).contiguous()

    def merge_strings(self, chars, nbytes, starts, lcps, counts, offsets):
        out = lcp_merge_strings(self.ctx, chars, nbytes, lcps, counts, offsets, char_start=starts,
                                stream=self.stream)
        return dict(chars=out["chars"], char_bytes=out["char_bytes"], offsets=out["offsets"], lengths=out["lengths"],
                    lcp=out["merged_lcp"])

    def no_strings(self):
        torch = self.torch
        return dict(chars=torch.zeros(1, dtype=torch.uint8, device=self.device), char_bytes=0,
                    offsets=torch.zeros(0, dtype=torch.int64, device=self.device),
                    lengths=self._e(0, torch.int32), lcp=self._e(0, torch.int32))

    def to_host(self, t, n=None):
        a = t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)
        if a.dtype == np.int32:
            a = a.view(np.uint32)
        a = a.astype(np.int64)
        return a if n is None else a[:n]


# ------------------------------------------------------------- the path ----
def sample_positions(sizes, p_global: int, factor: int = 2):
    """Per PE of `sizes` strings: the local indices SampleSplittersNumStringsPolicy
    samples (nr = min(factor (p-1), n_q), index floor(i n_q / (nr + 1)) in double
    arithmetic, samplingStrategies.hpp:57-89), as int64 arrays."""
    out = []
    for nq in sizes:
        nq = int(nq)
        nr = min(factor * (p_global - 1), nq)
        dist = float(nq) / float(nr + 1)
        out.append(np.floor(np.arange(1, nr + 1, dtype=np.float64) * dist).astype(np.int64))
    return out


def _pack_rows(*cols, blob=None):
    """One int64 message: the column lengths, the columns, then the blob bytes
    (padded to 8) viewed as int64 — one all-gather instead of one per column."""
    blob = np.zeros(0, np.uint8) if blob is None else np.ascontiguousarray(blob, np.uint8)
    padded = np.zeros((blob.size + 7) // 8 * 8, np.uint8)
    padded[:blob.size] = blob
    head = [len(cols), blob.size] + [int(np.asarray(c).size) for c in cols]
    parts = [np.asarray(head, np.int64)] + [np.asarray(c, np.int64).ravel() for c in cols] + [padded.view(np.int64)]
    return np.concatenate(parts)


def _unpack_rows(msg):
    """Inverse of _pack_rows: (list of int64 columns, uint8 blob)."""
    msg = np.ascontiguousarray(msg, np.int64)
    k, nb = int(msg[0]), int(msg[1])
    sizes = [int(x) for x in msg[2:2 + k]]
    at = 2 + k
    cols = []
    for m in sizes:
        cols.append(msg[at:at + m])
        at += m
    return cols, msg[at:].view(np.uint8)[:nb]


def depths():
    """The depth schedule of computeDistinguishingPrefixes: 8, 24, 40, 72, 136, ..."""
    yield 8
    i = 16
    while True:
        yield 8 + i
        i *= 2


class _Phases:
    """Wall-clock time per phase (after a device synchronisation), when asked."""

    def __init__(self, out):
        import time
        self.out, self.time = out, time
        self.t = time.perf_counter() if out is not None else 0.0

    def mark(self, name):
        if self.out is None:
            return
        try:
            import torch
            if torch.cuda.is_available():
                torch.cuda.synchronize()
        except ImportError:
            pass
        t = self.time.perf_counter()
        self.out[name] = self.out.get(name, 0.0) + (t - self.t) * 1e3
        self.t = t


def _partition(comm, be, strings, pb, order, trunc, sizes_local, p, p_local, q_first, pe_goff, factor, indexed):
    """Splitters from every PE's sample, each sample string cut to trunc(its
    local positions), gathered on all ranks and sorted; this rank's interval
    rows (computePartition, misc.hpp:531-587) and every rank's."""
    pos = sample_positions(sizes_local, p, factor)
    if p_local:
        flat = np.concatenate([pb[q] + pos[q] for q in range(p_local)])
        gidx = np.concatenate([pe_goff[q_first + q] + pos[q] for q in range(p_local)])
    else:
        flat = gidx = np.zeros(0, np.int64)
    ids = be.take(order, flat) if flat.size else np.zeros(0, np.int64)
    tr = trunc(flat) if flat.size else np.zeros(0, np.int64)
    schars, soffs, slens, sbytes = be.pack(strings, ids, tr)
    # every rank's (lengths, offsets, global indices, bytes) in one all-gather
    msg = _pack_rows(slens, soffs, gidx, blob=np.asarray(be.chars_to_host(schars, sbytes), np.uint8))
    base, offs, lens_l, gidx_l, chars_l = 0, [], [], [], []
    for part in comm.allgather_np(msg):
        (ln, of, gi), cb = _unpack_rows(part)
        lens_l.append(ln)
        offs.append(of + base)
        gidx_l.append(gi)
        chars_l.append(cb)
        base += cb.size
    gchars = np.concatenate(chars_l) if chars_l else np.zeros(0, np.uint8)
    goffs = np.concatenate(offs)
    glens = np.concatenate(lens_l)
    ggidx = np.concatenate(gidx_l)
    S = int(glens.size)
    sample = be.arena_from(be.chars_from_host(gchars), goffs, glens, gchars.size)
    nspl = min(p - 1, S)
    if nspl:
        sorted_ids = np.asarray(be.sort_arena(sample), np.int64)
        step = S // (nspl + 1)
        spl_ids = sorted_ids[np.arange(1, nspl + 1, dtype=np.int64) * step]
    else:
        spl_ids = np.zeros(0, np.int64)
    pchars, poffs, plens, pbytes = be.pack(sample, spl_ids, None)
    spl = be.arena_from(pchars, poffs, plens, pbytes)
    iv_local = be.partition_search(strings, pb, order, spl, ggidx[spl_ids], p, pe_goff[q_first:q_first + p_local],
                                   indexed)
    iv_all = np.concatenate(comm.allgather_np(np.asarray(iv_local).ravel())).reshape(p, p)
    return iv_local, iv_all


def _exchange(comm, be, strings, pb, order, lcp, dp, p, p_all, p_local, q_first, iv_local, iv_all, compress_lcps,
              ph):
    """Receive containers of [lcp, dp) + NUL per string to every PE, across
    ranks (alltoall.hpp:910-1008), regrouped by receiving PE; returns the
    regroup plan, the received bytes, starts and LCPs, the strings and bytes
    received, and per local receiving PE the strings and bucket offsets of
    every source PE."""
    snd = be.bucket_send(strings, pb, order, lcp, dp, p, q_first, iv_local)
    ph.mark("bucket_send")
    per_r = snd["counts"].sum(axis=1)                    # strings per receiver from this rank
    rbeg = np.concatenate([[0], np.cumsum(per_r)])
    cbeg = snd["char_begin"]
    firsts = np.concatenate([[0], np.cumsum(p_all)])
    s_str = [int(rbeg[firsts[t + 1]] - rbeg[firsts[t]]) for t in range(comm.world)]
    s_byte = [int(cbeg[firsts[t + 1]] - cbeg[firsts[t]]) for t in range(comm.world)]
    # to every rank: (strings, bytes) of each of its receivers from this rank
    nbytes_r = np.diff(cbeg)
    meta = [np.stack([per_r[firsts[t]:firsts[t + 1]], nbytes_r[firsts[t]:firsts[t + 1]]]).T.ravel()
            for t in range(comm.world)]
    rmeta = [m.reshape(-1, 2) for m in comm.alltoall_np(meta)]
    r_str = comm.alltoall_counts(s_str)
    r_byte = comm.alltoall_counts(s_byte)
    rchars = comm.alltoallv(snd["chars"], s_byte, r_byte)
    rstart = comm.alltoallv(snd["char_start"], s_str, r_str)
    if compress_lcps:
        # sendLcps with compressLcps (alltoall.hpp:406-425): each rank's run of
        # LCPs varint-coded (writeRanges), the bytes exchanged, and all that
        # arrives decoded as one sequence (varint codes are self-delimiting)
        lbytes, per_rank = be.varint_encode(snd["lcp"], s_str)
        r_lb = comm.alltoall_counts([int(x) for x in per_rank])
        got = comm.alltoallv(lbytes, [int(x) for x in per_rank], r_lb)
        rlcp = be.varint_decode(got, int(sum(r_str)))
    else:
        rlcp = comm.alltoallv(snd["lcp"], s_str, r_str)
    ph.mark("exchange")
    # regroup [sender rank][receiver] -> [receiver][sender rank]
    src_str = np.concatenate([[0], np.cumsum(r_str)])
    src_byte = np.concatenate([[0], np.cumsum(r_byte)])
    blocks, dstr, dbyte = [], 0, 0
    for r in range(p_local):
        for s in range(comm.world):
            ns_, nb_ = int(rmeta[s][r, 0]), int(rmeta[s][r, 1])
            so = int(src_str[s] + rmeta[s][:r, 0].sum())
            bo = int(src_byte[s] + rmeta[s][:r, 1].sum())
            blocks.append([so, dstr, ns_, bo, dbyte, nb_])
            dstr += ns_
            dbyte += nb_
    nrecv = dstr
    my = slice(q_first, q_first + p_local)
    counts = iv_all[:, my].T.copy()                                            # [r_local, q]
    starts = np.concatenate([np.zeros((p, 1), np.int64), np.cumsum(iv_all, axis=1)], axis=1)
    offsets = starts[:, my].T.copy()                                           # [r_local, q]
    return blocks, rchars, rstart, rlcp, nrecv, dbyte, counts, offsets


def sort(comm: Comm, be, strings, part_begin, sampler: int = 0, factor: int = 2, phases=None,
         compress_lcps: bool = False, golomb: bool = False, fused: bool = True):
    """This rank's part of DistributedPrefixDoublingSort::sort.  strings: the
    backend's arena of this rank's strings; part_begin: p_local + 1 PE bounds.
    phases (dict, optional) receives milliseconds per phase.  fused: with one
    rank, the one-GPU path (False: the staged path with its exchanges, as
    with several ranks).  golomb: the
    hashes of every round cross as Golomb/delta-coded blocks, the
    sequentialGolombEncoding policy (AllToAllHashesGolomb,
    bloomfilter.hpp:164-243): each rank's hash records sorted (ips4o::sort,
    :1512), one block per owning rank with b = getB(2^64 - 1 / ranks, count),
    read back block after block by the owner."""
    ph = _Phases(phases)
    indexed = sampler == 2
    pb = np.asarray(part_begin, np.int64)
    p_local = len(pb) - 1
    n = int(pb[-1])
    sizes_local = np.diff(pb)
    sizes_all = comm.allgather_np(sizes_local)
    p_all = [len(x) for x in sizes_all]
    p = sum(p_all)
    q_first = sum(p_all[:comm.rank])
    pe_sizes = np.concatenate(sizes_all)
    pe_goff = np.concatenate([[0], np.cumsum(pe_sizes)]).astype(np.int64)
    res = dict(part_begin=pb, p_global=p, q_first=q_first)

    ph.mark("setup")
    if fused and comm.world == 1 and p > 1 and factor == 2 and hasattr(be, "fused_sort"):
        # one rank holds every PE: nothing crosses GPUs, so the one-GPU path
        # (one global sort, DP rounds over it, projections for the exchange)
        # gives this rank's results directly
        out = be.fused_sort(strings, pb, sampler)
        res.update(out)
        res["recv_total"] = int(np.asarray(out["recv_counts"]).sum())
        ph.mark("fused")
        return res

    # local sort (prefix_doubling.hpp:228)
    order, lcp = be.local_sort(strings, pb)
    res["local_order"] = order
    ph.mark("local_sort")
    if p == 1:  # prefix_doubling.hpp:236
        res["recv_counts"] = np.zeros(p_local, np.int64)
        return res

    # 1. distinguishing prefixes (prefix_doubling.hpp:157-198)
    dp = be.new_dp(n)
    state = None
    rounds = 0
    for depth in depths():
        state_out, hpos, hval = be.dp_classify(strings, order, lcp, state, depth, dp)
        if golomb:
            hval, hpos = be.hash_sort(hval, hpos)  # the owner groups then hold ascending hashes
        r_hval, r_hpos, counts = be.hash_route(hval, hpos, comm.world)
        recv = comm.alltoall_counts(counts)
        if golomb:
            bs = [be.golomb_param_hashes(c, comm.world) if c else 1 for c in counts]
            words, rw = be.golomb_encode(r_hval, counts, bs)
            wrecv = comm.alltoall_counts(rw)
            got, bc = be.golomb_decode(comm.alltoallv(words, rw, wrecv))
            if bc != [c for c in recv if c]:
                raise RuntimeError("Golomb blocks do not match the hash counts sent")
        else:
            got = comm.alltoallv(r_hval, counts, recv)
        dup = be.hash_dups(got)
        back = comm.alltoallv(dup, recv, counts)
        cand = be.dp_apply(r_hpos, back, state_out)
        state = state_out
        rounds += 1
        if comm.allreduce_sum(cand) == 0:
            break
    res["dp"] = dp
    res["dp_rounds"] = rounds
    ph.mark("dp")

    # 2. splitters (misc.hpp:531-587)
    iv_local, iv_all = _partition(comm, be, strings, pb, order, lambda flat: be.take(dp, flat), sizes_local, p,
                                  p_local, q_first, pe_goff, factor, indexed)
    res["intervals"] = np.asarray(iv_local, np.int64)
    ph.mark("partition")

    # 3. string exchange (alltoall.hpp:910-1008) and merge (merging.hpp:66-123)
    blocks, rchars, rstart, rlcp, nrecv, dbyte, counts, offsets = _exchange(
        comm, be, strings, pb, order, lcp, dp, p, p_all, p_local, q_first, iv_local, iv_all, compress_lcps, ph)
    res["recv_counts"] = counts.sum(axis=1)
    res["recv_total"] = nrecv
    if nrecv:
        mchars, mstart, mlcp = be.regroup(blocks, rchars, rstart, rlcp, nrecv, dbyte)
        ph.mark("regroup")
        res.update(be.merge(mchars, dbyte, mstart, mlcp, counts, offsets))
        ph.mark("merge")
    else:
        res.update(perm_index=np.zeros(0, np.int64), perm_pe=np.zeros(0, np.int64), merged_lcp=np.zeros(0, np.int64))
    return res


def merge_sort(comm: Comm, be, strings, part_begin, factor: int = 2, phases=None, compress_lcps: bool = False):
    """This rank's part of DistributedMergeSort::sort
    (lcp_aware_number_string_splitting.hpp:184-290) with
    SampleSplittersNumStringsPolicy: local sort, getAvgLcp over all PEs
    (misc.hpp:68-87), splitters from samples cut to 200 (avg + 5) bytes
    (misc.hpp:473-531 on 100 * avg, :238), whole strings exchanged
    prefix-compressed (DP = length), merged and decompressed on the receiving
    side (extendPrefix).  Returns per local receiving PE, back to back, the
    strings whole (chars, offsets, lengths), their LCPs (0 at each PE start),
    recv_counts, plus local_order, intervals and avg_lcp.  Byte-identical
    strings are interchangeable in this output."""
    ph = _Phases(phases)
    pb = np.asarray(part_begin, np.int64)
    p_local = len(pb) - 1
    n = int(pb[-1])
    sizes_local = np.diff(pb)
    sizes_all = comm.allgather_np(sizes_local)
    p_all = [len(x) for x in sizes_all]
    p = sum(p_all)
    q_first = sum(p_all[:comm.rank])
    pe_goff = np.concatenate([[0], np.cumsum(np.concatenate(sizes_all))]).astype(np.int64)
    res = dict(part_begin=pb, p_global=p, q_first=q_first)
    ph.mark("setup")
    order, lcp = be.local_sort(strings, pb)
    res["local_order"] = order
    ph.mark("local_sort")
    # getAvgLcp: the local LCP arrays (0 at each PE start) over all strings
    total_lcp = comm.allreduce_sum(be.lcp_sum(lcp, n))
    total_n = comm.allreduce_sum(n)
    avg = total_lcp // total_n if total_n else 0
    res["avg_lcp"] = avg
    cut = 2 * (100 * (avg + 5))
    iv_local, iv_all = _partition(comm, be, strings, pb, order, lambda flat: np.full(flat.size, cut, np.int64),
                                  sizes_local, p, p_local, q_first, pe_goff, factor, False)
    res["intervals"] = np.asarray(iv_local, np.int64)
    ph.mark("partition")
    dp = be.lengths_in_order(strings, order)
    blocks, rchars, rstart, rlcp, nrecv, dbyte, counts, offsets = _exchange(
        comm, be, strings, pb, order, lcp, dp, p, p_all, p_local, q_first, iv_local, iv_all, compress_lcps, ph)
    res["recv_counts"] = counts.sum(axis=1)
    res["recv_total"] = nrecv
    if nrecv:
        mchars, mstart, mlcp = be.regroup(blocks, rchars, rstart, rlcp, nrecv, dbyte)
        ph.mark("regroup")
        res.update(be.merge_strings(mchars, dbyte, mstart, mlcp, counts, offsets))
        ph.mark("merge")
    else:
        res.update(be.no_strings())
    return res
