"""Host backend for the distributed path (distributed-string-sorting_b200/dist.py):
the same methods as dist.GpuBackend, computed with the oracle and numpy, so
that the collectives and the host logic between them run on CPU ranks (gloo).
Test infrastructure only."""
import numpy as np

M64 = (1 << 64) - 1


class HostArena:
    def __init__(self, chars, offsets, lengths, nbytes):
        self.chars = np.ascontiguousarray(chars, np.uint8)
        self.offsets = np.ascontiguousarray(offsets, np.uint64)
        self.lengths = np.ascontiguousarray(lengths, np.uint32)
        self.char_bytes = int(nbytes)

    @property
    def n(self):
        return int(self.lengths.size)

    def get(self, i):
        o, l = int(self.offsets[i]), int(self.lengths[i])
        return self.chars[o:o + l].tobytes()


def pack_list(strs):
    lens = np.array([len(s) for s in strs], np.int64)
    offs = np.zeros(len(strs), np.int64)
    if len(strs):
        offs[1:] = np.cumsum(lens + 1)[:-1]
    blob = b"".join(s + b"\0" for s in strs)
    chars = np.frombuffer(blob + b"\0" * 64, np.uint8).copy()
    return chars, offs, lens, len(blob)


class OracleBackend:
    def __init__(self, orc):
        self.orc = orc

    def _s(self, a):
        return self.orc.Strings(a.chars, np.asarray(a.offsets, np.uint64), np.asarray(a.lengths, np.uint32))

    def local_sort(self, a, pb):
        order, lcp = self.orc.local_sort(self._s(a), np.asarray(pb, np.uint64))
        return order.astype(np.int64), lcp.astype(np.int64)

    def new_dp(self, n):
        return np.zeros(n, np.int64)

    def dp_classify(self, a, order, lcp, state, depth, dp):
        n = a.n
        cand = np.ones(n, bool) if state is None else np.asarray(state).astype(bool)
        lens = np.asarray(a.lengths, np.int64)[order]
        eos = cand & (depth > lens)
        dp[eos] = lens[eos]
        alive = cand & ~eos
        dp[alive] = depth
        prev_c = np.r_[False, cand[:-1]]
        dup = alive & prev_c & (lcp >= depth)
        hashed = alive & ~dup
        nxt = np.r_[cand[1:] & (lcp[1:] >= depth), False]
        root = hashed & nxt
        state_out = (dup | root).astype(np.uint8)
        hpos = np.nonzero(hashed)[0].astype(np.int64)
        hval = np.array([self.orc.xxh64(a.get(int(order[i]))[:depth]) % M64 for i in hpos], np.uint64)
        return state_out, hpos, hval

    def hash_route(self, hval, hpos, nowner):
        owner = np.array([(int(h) * nowner) >> 64 for h in hval], np.int64)
        perm = np.argsort(owner, kind="stable")
        counts = np.bincount(owner, minlength=nowner) if owner.size else np.zeros(nowner, np.int64)
        return hval[perm], hpos[perm], [int(c) for c in counts]

    def hash_sort(self, hval, hpos):
        perm = np.argsort(np.asarray(hval, np.uint64), kind="stable")
        return np.asarray(hval, np.uint64)[perm], np.asarray(hpos)[perm]

    def golomb_param_hashes(self, count, p):
        return self.orc.golomb_param_hashes(int(count), int(p))

    def golomb_encode(self, hval, counts, bs):
        words, rw = self.orc.golomb_encode(np.asarray(hval, np.uint64), counts, bs)
        return words, [int(x) for x in rw]

    def golomb_decode(self, words):
        vals, bc = self.orc.golomb_decode(np.asarray(words, np.uint64))
        return vals, [int(x) for x in bc]

    def hash_dups(self, got):
        got = np.asarray(got)
        if got.size == 0:
            return np.zeros(0, np.uint8)
        _, inv, cnt = np.unique(got, return_inverse=True, return_counts=True)
        return (cnt[inv.ravel()] >= 2).astype(np.uint8)

    def dp_apply(self, hpos, dup, state):
        state[np.asarray(hpos)[np.asarray(dup).astype(bool)]] = 1
        return int(state.sum())

    def take(self, t, idx):
        return np.asarray(t)[np.asarray(idx, np.int64)].astype(np.int64)

    def pack(self, a, ids, trunc=None):
        strs = []
        for j, i in enumerate(ids):
            s = a.get(int(i))
            if trunc is not None:
                s = s[:int(trunc[j])]
            strs.append(s)
        return pack_list(strs)

    def chars_to_host(self, chars, nbytes):
        return np.asarray(chars[:nbytes], np.uint8)

    def chars_from_host(self, a):
        return np.concatenate([np.asarray(a, np.uint8), np.zeros(64, np.uint8)])

    def arena_from(self, chars, offsets, lengths, nbytes):
        return HostArena(chars, offsets, lengths, nbytes)

    def sort_arena(self, a):
        order, _ = self.orc.local_sort(self._s(a), np.array([0, a.n], np.uint64))
        return order.astype(np.int64)

    @staticmethod
    def _scmp(x, y):
        return (x > y) - (x < y)

    def partition_search(self, a, pb, order, spl, spl_index, p_global, pe_index, indexed):
        """binarySearch / binarySearchIndexed (misc.hpp:310-374) per (PE, splitter)."""
        p_local = len(pb) - 1
        iv = np.zeros((p_local, p_global), np.int64)
        nspl = spl.n
        for q in range(p_local):
            base, nq = int(pb[q]), int(pb[q + 1] - pb[q])
            pos = []
            for k in range(nspl):
                sk = spl.get(k)
                left, right, hit = 0, nq, None
                while left != right:
                    d = (right - left) // 2
                    res = self._scmp(a.get(int(order[base + left + d])), sk)
                    if res == 0 and indexed:
                        diff = (left + d + int(pe_index[q]) - int(spl_index[k])) & 0xFFFFFFFF
                        res = diff - (1 << 32) if diff >= (1 << 31) else diff
                    if res < 0:
                        left = left + d + 1
                    elif res == 0:
                        hit = left + d
                        break
                    else:
                        right = left + d
                pos.append(left if hit is None else hit)
            prev = 0
            for r in range(p_global):
                cur = pos[r] if r < nspl else nq
                iv[q, r] = cur - prev
                prev = cur
        return iv

    def bucket_send(self, a, pb, order, lcp, dp, p_global, q_first, iv_local):
        p_local = len(pb) - 1
        chars, starts, lcps = [], [], []
        counts = np.zeros((p_global, p_local), np.int64)
        char_begin = [0]
        pos = 0
        bounds = np.concatenate([np.zeros((p_local, 1), np.int64), np.cumsum(iv_local, axis=1)], axis=1)
        for r in range(p_global):
            rstart = pos
            for q in range(p_local):
                b0, b1 = int(bounds[q, r]), int(bounds[q, r + 1])
                counts[r, q] = b1 - b0
                for i in range(b0, b1):
                    g = int(pb[q]) + i
                    l = 0 if i == b0 else int(lcp[g])
                    s = a.get(int(order[g]))[l:int(dp[g])]
                    starts.append(pos - rstart)
                    lcps.append(l)
                    chars.append(s + b"\0")
                    pos += len(s) + 1
            char_begin.append(pos)
        blob = b"".join(chars)
        return dict(chars=np.frombuffer(blob, np.uint8).copy(), char_start=np.array(starts, np.int64),
                    lcp=np.array(lcps, np.int64), char_begin=np.array(char_begin, np.int64), counts=counts)

    def regroup(self, blocks, chars, starts, lcps, n, nbytes):
        dchars = np.zeros(nbytes + 64, np.uint8)
        dstart = np.zeros(n, np.int64)
        dlcp = np.zeros(n, np.int64)
        for so, do, ns, bo, dbo, nb in blocks:
            dchars[dbo:dbo + nb] = np.asarray(chars)[bo:bo + nb]
            dstart[do:do + ns] = np.asarray(starts)[so:so + ns] + dbo
            dlcp[do:do + ns] = np.asarray(lcps)[so:so + ns]
        return dchars, dstart, dlcp

    def varint_encode(self, values, range_counts):
        return self.orc.varint_encode(values, range_counts)

    def varint_decode(self, data, n):
        return self.orc.varint_decode(data, n)

    def merge(self, chars, nbytes, starts, lcps, counts, offsets):
        out = {k: [] for k in ("perm_index", "perm_pe", "merged_lcp")}
        k = 0
        for r in range(counts.shape[0]):
            m = int(counts[r].sum())
            if m == 0:
                continue
            b0 = int(starts[k])
            b1 = int(starts[k + m - 1])
            while chars[b1] != 0:
                b1 += 1
            idx, pe, ml, _ = self.orc.merge(np.asarray(chars[b0:b1 + 1]), np.asarray(lcps[k:k + m]), counts[r],
                                            offsets[r])
            out["perm_index"].append(idx)
            out["perm_pe"].append(pe)
            out["merged_lcp"].append(ml)
            k += m
        return {key: (np.concatenate(v).astype(np.int64) if v else np.zeros(0, np.int64)) for key, v in out.items()}

    def lcp_sum(self, lcp, n):
        return int(np.asarray(lcp, np.int64)[:n].sum())

    def lengths_in_order(self, a, order):
        return np.asarray(a.lengths, np.int64)[np.asarray(order, np.int64)]

    def merge_strings(self, chars, nbytes, starts, lcps, counts, offsets):
        """The merge, then every run's strings with their prefixes restored
        (extendPrefix, strings/stringcontainer.hpp:248-333), in merged order."""
        m = self.merge(chars, nbytes, starts, lcps, counts, offsets)
        chars, starts, lcps = np.asarray(chars), np.asarray(starts), np.asarray(lcps)
        full, run_pos, k = [], {}, 0
        for r in range(counts.shape[0]):
            for q in range(counts.shape[1]):
                run_pos[(r, q)] = k
                prev = b""
                for _ in range(int(counts[r, q])):
                    b0 = b1 = int(starts[k])
                    while chars[b1] != 0:
                        b1 += 1
                    cur = prev[:int(lcps[k])] + chars[b0:b1].tobytes()
                    full.append(cur)
                    prev = cur
                    k += 1
        out, t = [], 0
        for r in range(counts.shape[0]):
            for _ in range(int(counts[r].sum())):
                q, i = int(m["perm_pe"][t]), int(m["perm_index"][t])
                out.append(full[run_pos[(r, q)] + i - int(offsets[r, q])])
                t += 1
        oc, oo, ol, nb = pack_list(out)
        return dict(chars=oc, char_bytes=nb, offsets=oo, lengths=ol, lcp=m["merged_lcp"])

    def no_strings(self):
        z = np.zeros(0, np.int64)
        return dict(chars=np.zeros(1, np.uint8), char_bytes=0, offsets=z, lengths=z, lcp=z)

    def to_host(self, t, n=None):
        a = np.asarray(t).astype(np.int64)
        return a if n is None else a[:n]
