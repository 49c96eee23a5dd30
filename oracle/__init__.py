"""ORACLE — test infrastructure only.

ctypes wrappers over oracle/liboracle.so (the CPU restatement of the
reference's prefix-doubling path, oracle/oracle.cpp) and, where built, the
pieces of the reference compiled from its own sources (oracle/_ref/).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs may use this
package, and only as the checker or the timed CPU baseline; the product never
calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF = os.path.join(HERE, "_ref", "libref.so")
REF_DP = os.path.join(HERE, "_ref", "libref_dp.so")

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_I = ctypes.c_int

_lib = None
_ref = None
_ref_dp = None


REF_EXE = os.path.join(HERE, "_ref", "prefix_doubling")
REF_MP = os.path.join(HERE, "_ref", "ref_mp")


def reference_tree():
    """The reference checkout to compile oracle/_ref from: $DSSS_REFERENCE, else
    the read-only checkout this build container mounts, else None (a machine
    without it uses the prebuilt oracle/_ref)."""
    for cand in (os.environ.get("DSSS_REFERENCE"), "/root/reference"):
        if cand and os.path.exists(os.path.join(cand, "src", "hash", "xxhash.hpp")):
            return cand
    return None


def build():
    """Compiles liboracle.so (and oracle/_ref when the reference tree is present)."""
    cmd = ["make", "-s", "-C", HERE]
    tree = reference_tree()
    if tree:
        cmd.append("REF=" + tree)
    subprocess.run(cmd, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_xxh64.restype = _U64
        L.oracle_xxh64.argtypes = [_P, _U64]
        L.oracle_local_sort.restype = None
        L.oracle_local_sort.argtypes = [_P, _P, _P, _U64, _U32, _P, _P, _P]
        L.oracle_dp.restype = None
        L.oracle_dp.argtypes = [_P, _P, _P, _U64, _U32, _P, _P, _P, _P, _P, _U32, _P]
        L.oracle_partition.restype = None
        L.oracle_partition.argtypes = [_P, _P, _P, _U64, _U32, _P, _P, _P, _U32, _I, _P]
        L.oracle_exchange.restype = _I
        L.oracle_exchange.argtypes = [_P, _P, _P, _U64, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.oracle_merge.restype = _I
        L.oracle_merge.argtypes = [_P, _U64, _P, _U64, _U32, _P, _P, _P, _P, _P, _P]
        L.oracle_pd_sort.restype = _I
        L.oracle_pd_sort.argtypes = [_P, _P, _P, _U64, _U32, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.oracle_ms_sort.restype = _I
        L.oracle_ms_sort.argtypes = [_P, _P, _P, _U64, _U32, _P, _P, _P, _P, _P, _P, _P, _P]
        L.oracle_gen_dn.restype = _I
        L.oracle_gen_dn.argtypes = [_U64, _U32, _U32, _U32, _U32, ctypes.c_double, _U64, _P, _P, _P, _P]
        L.oracle_hq_sort.restype = _I
        L.oracle_hq_sort.argtypes = [_P, _P, _P, _U64, _U32, _P, _U64, _P, _P]
        _lib = L
    return _lib


def gen_dn(n, L, k, seed, long_len=0, long_k=0, frac_long=0.0):
    """The D/N-rule input, generated by the oracle's own restatement of the
    rule (no product code): a Strings of n strings, NUL-terminated back to
    back."""
    L_ = lib()
    tot = ctypes.c_uint64(0)
    rc = L_.oracle_gen_dn(n, L, k, long_len, long_k, frac_long, seed, None, None, None, ctypes.byref(tot))
    assert rc == 0, rc
    chars = np.zeros(tot.value + 64, np.uint8)
    offsets = np.zeros(max(n, 1), np.uint64)
    lengths = np.zeros(max(n, 1), np.uint32)
    rc = L_.oracle_gen_dn(n, L, k, long_len, long_k, frac_long, seed, _p(chars), _p(offsets), _p(lengths),
                          ctypes.byref(tot))
    assert rc == 0, rc
    s = Strings(chars, offsets[:n], lengths[:n])
    s.char_bytes = tot.value
    return s


def write_lines(s, path):
    """Writes the strings one per line (the reference's --generator 2 input:
    FileDistributer turns every newline into the NUL terminator).  The strings
    must be back to back, NUL-terminated, as gen_dn makes them."""
    chars = s.chars[:s.char_bytes].copy()
    chars[chars == 0] = 10
    with open(path, "wb") as f:
        f.write(memoryview(chars))


def ref_exe_available() -> bool:
    return os.path.exists(REF_EXE)


def run_reference_pd(path, np_ranks, iterations, extra=(), timeout=3600, env=None):
    """Runs the reference's own prefix_doubling executable (compiled into
    oracle/_ref over the process-based MPI stand-in) on a file of strings with
    np_ranks ranks: ``--generator 2 --path <file> --strongScaling``.  Returns
    the per-iteration `sorting_overall` time in seconds (its maxTime RESULT
    value: the slowest rank, src/util/timer.hpp) and the output."""
    e = dict(os.environ)
    e.update(env or {})
    e["DSSS_MPI_NP"] = str(np_ranks)
    cmd = [REF_EXE, "--generator", "2", "--path", path, "--strongScaling", "--numberOfIterations",
           str(iterations), *extra]
    out = subprocess.run(cmd, env=e, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"reference prefix_doubling failed ({out.returncode}): {out.stderr[-2000:]}")
    times = {}
    for line in out.stdout.splitlines():
        if not line.startswith("RESULT") or "operation=sorting_overall" not in line or "type=maxTime" not in line:
            continue
        kv = dict(t.split("=", 1) for t in line.split()[1:] if "=" in t)
        times[int(kv["iteration"])] = int(kv["value"]) * 1e-9
    return [times[i] for i in sorted(times)], out.stdout


def ref_mp_available() -> bool:
    return os.path.exists(REF_MP)


def run_reference_mp(mode, s, pb, timeout=600):
    """Runs the reference's own distributed sorter (oracle/ref_bridge_mp.cpp:
    mode "pd", "pdi", "ms" or "hq") with one process per PE over the
    process-based MPI stand-in, PE q holding strings pb[q]..pb[q+1] of `s`.
    Returns one dict per rank with that mode's arrays (see the bridge)."""
    import tempfile
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    raw = s.raw()
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        with open(inp, "wb") as f:
            f.write(np.array([s.n, p], np.uint64).tobytes())
            f.write(pb.tobytes())
            f.write(np.array([len(raw)], np.uint64).tobytes())
            f.write(raw)
        e = dict(os.environ)
        e["DSSS_MPI_NP"] = str(p)
        e.setdefault("DSSS_MPI_ARENA_GB", "2")
        out = subprocess.run([REF_MP, mode, inp, os.path.join(td, "out")], env=e, capture_output=True, text=True,
                             timeout=timeout)
        if out.returncode != 0:
            raise RuntimeError(f"ref_mp {mode} failed ({out.returncode}): {out.stderr[-2000:]}")
        names = {"pd": ("order", "lcp", "dp", "intervals", "perm"), "pdi": ("order", "lcp", "dp", "intervals", "perm"),
                 "ms": ("bytes", "lcp"), "hq": ("bytes",)}[mode]
        res = []
        for q in range(p):
            with open(os.path.join(td, f"out.{q}"), "rb") as f:
                buf = f.read()
            pos, d = 0, {}
            for nm in names:
                c = int(np.frombuffer(buf, np.uint64, 1, pos)[0])
                d[nm] = np.frombuffer(buf, np.uint64, c, pos + 8).copy()
                pos += 8 + 8 * c
            res.append(d)
    return res


def ref_available() -> bool:
    return os.path.exists(REF)


def ref_dp_available() -> bool:
    return os.path.exists(REF_DP)


def ref():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF)
        L.ref_xxh64.restype = _U64
        L.ref_xxh64.argtypes = [_P, _U64]
        L.ref_radixsort_ci3.restype = _I
        L.ref_radixsort_ci3.argtypes = [_P, _U64, _U64, _P, _P]
        L.ref_lcp_merge.restype = _I
        L.ref_lcp_merge.argtypes = [_P, _U64, _P, _U64, _U32, _P, _P, _P, _P, _P, _P]
        L.ref_golomb_param.restype = _U64
        L.ref_golomb_param.argtypes = [_U64, _U64]
        L.ref_golomb_block.restype = ctypes.c_int64
        L.ref_golomb_block.argtypes = [_P, _U64, _U64, _P, _U64]
        L.ref_golomb_unblock.restype = ctypes.c_int64
        L.ref_golomb_unblock.argtypes = [_P, _U64, _P, _U64]
        _ref = L
    return _ref


def ref_dp():
    global _ref_dp
    if _ref_dp is None:
        L = ctypes.CDLL(REF_DP)
        L.ref_dp_single_pe.restype = _I
        L.ref_dp_single_pe.argtypes = [_P, _U64, _U64, _P, _P, _P]
        _ref_dp = L
    return _ref_dp


def _p(a):
    return a.ctypes.data if a is not None else None


class Strings:
    """Host strings for the oracle: chars (uint8 with >= 8 bytes of slack), offsets, lengths."""

    def __init__(self, chars, offsets, lengths):
        self.chars = np.ascontiguousarray(chars, dtype=np.uint8)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
        self.n = int(self.offsets.shape[0])

    @classmethod
    def from_host(cls, hs):
        return cls(hs.chars, hs.offsets, hs.lengths)

    def args(self):
        return (_p(self.chars), _p(self.offsets), _p(self.lengths), self.n)

    def get(self, i):
        o, l = int(self.offsets[i]), int(self.lengths[i])
        return self.chars[o:o + l].tobytes()

    def raw(self, ids=None):
        """NUL-terminated back-to-back layout (the reference's raw string vector)."""
        ids = range(self.n) if ids is None else ids
        return b"".join(self.get(int(i)) + b"\0" for i in ids)


def xxh64(data: bytes) -> int:
    buf = np.frombuffer(data + b"\0" * 16, dtype=np.uint8)
    return int(lib().oracle_xxh64(_p(buf), len(data)))


def local_sort(s: Strings, pb):
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    order = np.zeros(max(s.n, 1), np.uint64)
    lcp = np.zeros(max(s.n, 1), np.uint64)
    lib().oracle_local_sort(*s.args(), len(pb) - 1, _p(pb), _p(order), _p(lcp))
    return order[:s.n], lcp[:s.n]


def dp_rounds(s: Strings, pb, order, lcp, max_rounds=64):
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    order = np.ascontiguousarray(order, dtype=np.uint64)
    lcp = np.ascontiguousarray(lcp, dtype=np.uint64)
    dp = np.zeros(max(s.n, 1), np.uint64)
    counts = np.zeros(max_rounds, np.uint64)
    rounds = ctypes.c_uint32(0)
    lib().oracle_dp(*s.args(), len(pb) - 1, _p(pb), _p(order), _p(lcp), _p(dp), _p(counts), max_rounds,
                    ctypes.byref(rounds))
    return dp[:s.n], counts[:rounds.value]


def partition(s: Strings, pb, order, dp, indexed=False, factor=2):
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    iv = np.zeros(p * p, np.uint64)
    order = np.ascontiguousarray(order, np.uint64)
    dp = np.ascontiguousarray(dp, np.uint64)
    lib().oracle_partition(*s.args(), p, _p(pb), _p(order), _p(dp), factor, 1 if indexed else 0, _p(iv))
    return iv.reshape(p, p)


def exchange(s: Strings, pb, order, lcp, dp, intervals):
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    keep = [np.ascontiguousarray(x, np.uint64).ravel() for x in (order, lcp, dp, intervals)]
    args = (*s.args(), p, _p(pb), *(_p(x) for x in keep))
    tot = ctypes.c_uint64(0)
    lib().oracle_exchange(*args, ctypes.byref(tot), None, None, None, None, None, None, None)
    n = s.n
    out = dict(chars=np.zeros(tot.value + 1, np.uint8), char_begin=np.zeros(p + 1, np.uint64),
               lcp=np.zeros(max(n, 1), np.uint64), index=np.zeros(max(n, 1), np.uint64),
               pe=np.zeros(max(n, 1), np.uint64), counts=np.zeros(p * p, np.uint64), offsets=np.zeros(p * p, np.uint64))
    lib().oracle_exchange(*args, ctypes.byref(tot), _p(out["chars"]), _p(out["char_begin"]), _p(out["lcp"]),
                          _p(out["index"]), _p(out["pe"]), _p(out["counts"]), _p(out["offsets"]))
    out["chars"] = out["chars"][:tot.value]
    for k in ("lcp", "index", "pe"):
        out[k] = out[k][:n]
    out["counts"] = out["counts"].reshape(p, p)
    out["offsets"] = out["offsets"].reshape(p, p)
    return out


def merge(chars, lcps, counts, offsets):
    """The oracle's loser-tree merge of one PE's receive container."""
    chars = np.ascontiguousarray(chars, np.uint8)
    lcps = np.ascontiguousarray(lcps, np.uint64)
    n = lcps.size
    p = len(counts)
    o = [np.zeros(max(n, 1), np.uint64) for _ in range(4)]
    counts = np.ascontiguousarray(counts, np.uint64)
    offsets = np.ascontiguousarray(offsets, np.uint64)
    rc = lib().oracle_merge(_p(chars), chars.size, _p(lcps), n, p, _p(counts), _p(offsets), *(_p(x) for x in o))
    assert rc == 0, rc
    return tuple(x[:n] for x in o)


def pd_sort(s: Strings, pb, indexed=False):
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    n = s.n
    z = lambda: np.zeros(max(n, 1), np.uint64)
    o = dict(order=z(), lcp=z(), dp=z(), intervals=np.zeros(p * p, np.uint64), perm_index=z(), perm_pe=z(),
             merged_lcp=z(), old_lcp=z(), recv_counts=np.zeros(p, np.uint64))
    rc = lib().oracle_pd_sort(*s.args(), p, _p(pb), 1 if indexed else 0, _p(o["order"]), _p(o["lcp"]), _p(o["dp"]),
                              _p(o["intervals"]), _p(o["perm_index"]), _p(o["perm_pe"]), _p(o["merged_lcp"]),
                              _p(o["old_lcp"]), _p(o["recv_counts"]))
    assert rc == 0
    for k in ("order", "lcp", "dp", "perm_index", "perm_pe", "merged_lcp", "old_lcp"):
        o[k] = o[k][:n]
    o["intervals"] = o["intervals"].reshape(p, p)
    return o


def ms_sort(s: Strings, pb):
    """The merge-sort path (oracle_ms_sort): local sort, average LCP, splitters
    from samples truncated to 200 (avg + 5) bytes, whole strings exchanged and
    merged; source = string id of every output string, receiving PEs back to back."""
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    n = s.n
    z = lambda: np.zeros(max(n, 1), np.uint64)
    o = dict(order=z(), lcp=z(), intervals=np.zeros(p * p, np.uint64), source=z(), out_lcp=z(),
             recv_counts=np.zeros(p, np.uint64))
    avg = np.zeros(1, np.uint64)
    rc = lib().oracle_ms_sort(*s.args(), p, _p(pb), _p(o["order"]), _p(o["lcp"]), _p(o["intervals"]),
                              _p(o["source"]), _p(o["out_lcp"]), _p(o["recv_counts"]), _p(avg))
    assert rc == 0
    for k in ("order", "lcp", "source", "out_lcp"):
        o[k] = o[k][:n]
    o["intervals"] = o["intervals"].reshape(p, p)
    o["avg_lcp"] = int(avg[0])
    return o


HQ_SEED = 3469931  # HQuicksort.cpp:344: PE r seeds its generator with 3469931 + r


def hq_sort(s: Strings, pb, seed: int = HQ_SEED):
    """RQuick::sort as hQuicksort runs it (oracle_hq_sort): source = string id
    of every output string, PEs back to back; counts = strings per PE."""
    pb = np.ascontiguousarray(pb, dtype=np.uint64)
    p = len(pb) - 1
    n = s.n
    src = np.zeros(max(n, 1), np.uint64)
    counts = np.zeros(p, np.uint64)
    rc = lib().oracle_hq_sort(*s.args(), p, _p(pb), seed, _p(src), _p(counts))
    assert rc == 0
    return dict(source=src[:n], counts=counts)


def distribute_strings(data: bytes, p: int, max_size: int = 0):
    """distribute_strings (src/mpi/readInput.hpp:40-104) restated rank by rank:
    the raw vector every rank ends with.  Raises ValueError where the reference
    reads past a buffer (a rank r > 0 whose slice holds no newline, or an
    empty last slice)."""
    S = min(len(data), max_size) if max_size > 0 else len(data)
    local, larger = S // p, S % p
    sl = []
    for r in range(p):  # :57-69
        if r < larger:
            ln = local + 1
            off = ln * r
        else:
            ln = local
            off = larger * (local + 1) + (r - larger) * local
        res = bytearray(data[off:off + ln])
        fe = 0  # :76-79
        while fe < len(res) and res[fe] != 10:
            fe += 1
        for i in range(len(res)):  # :80-82
            if res[i] == 10:
                res[i] = 0
        sl.append((res, fe))
    out = []
    for r in range(p):
        res = bytearray(sl[r][0])
        if r + 1 < p:  # :84-91, the next rank's shift_left of first_end + 1 bytes
            nxt, nfe = sl[r + 1]
            if nfe >= len(nxt):
                raise ValueError("rank %d's slice holds no newline" % (r + 1))
            res += nxt[:nfe + 1]
        else:  # :92-96
            if not res:
                raise ValueError("empty last slice")
            if res[-1] != 0:
                res.append(0)
        if r > 0:  # :97-99
            res = res[sl[r][1] + 1:]
        out.append(bytes(res))
    return out


def varint_encode(values, range_counts):
    """Writer::PutVarint (src/encoding/integer_compression.hpp:66-140) for every
    value: 7 bits per byte, least significant first, the high bit on every byte
    but the last; ranges back to back with their byte counts
    (IntegerCompression::writeRanges, src/mpi/byte_encoder.hpp:31-53)."""
    out, per, k = bytearray(), [], 0
    vals = np.asarray(values).astype(np.int64)
    for c in range_counts:
        start = len(out)
        for v in vals[k:k + int(c)].tolist():
            while v >= 128:
                out.append((v & 0x7F) | 0x80)
                v >>= 7
            out.append(v)
        per.append(len(out) - start)
        k += int(c)
    return np.frombuffer(bytes(out), np.uint8).copy(), np.asarray(per, np.uint64)


def varint_decode(data, n):
    """Reader::decode (src/encoding/integer_compression.hpp) of n values."""
    vals, v, sh = [], 0, 0
    for b in np.asarray(data, np.uint8).tolist():
        v |= (b & 0x7F) << sh
        sh += 7
        if not b & 0x80:
            vals.append(v)
            v, sh = 0, 0
    if len(vals) != n or sh != 0:
        raise ValueError("not %d whole values" % n)
    return np.asarray(vals, np.int64)


# ------------------------------------------------------------ reference ----
def ref_xxh64(data: bytes) -> int:
    buf = np.frombuffer(data + b"\0", dtype=np.uint8)
    return int(ref().ref_xxh64(_p(buf), len(data)))


def ref_local_sort(strs):
    """radixsort_CI3 of the reference on a list of byte strings: (order, lcp)."""
    raw = np.frombuffer(b"".join(x + b"\0" for x in strs) + b"\0", dtype=np.uint8)
    n = len(strs)
    order = np.zeros(max(n, 1), np.uint64)
    lcp = np.zeros(max(n, 1), np.uint64)
    rc = ref().ref_radixsort_ci3(_p(raw), raw.size - 1, n, _p(order), _p(lcp))
    assert rc == 0, rc
    return order[:n], lcp[:n]


def ref_dp_single_pe(strs):
    """The reference's own computeDistinguishingPrefixes on one PE: (order, lcp, dp)."""
    raw = np.frombuffer(b"".join(x + b"\0" for x in strs) + b"\0", dtype=np.uint8)
    n = len(strs)
    order = np.zeros(max(n, 1), np.uint64)
    lcp = np.zeros(max(n, 1), np.uint64)
    dp = np.zeros(max(n, 1), np.uint64)
    rc = ref_dp().ref_dp_single_pe(_p(raw), raw.size - 1, n, _p(order), _p(lcp), _p(dp))
    assert rc == 0, rc
    return order[:n], lcp[:n], dp[:n]


def ref_lcp_merge(chars, lcps, recv_counts, recv_offsets):
    """LcpStringLoserTree_ of the reference on one PE's receive container."""
    chars = np.ascontiguousarray(chars, np.uint8)
    lcps = np.ascontiguousarray(lcps, np.uint64)
    n = lcps.size
    p = len(recv_counts)
    o = [np.zeros(max(n, 1), np.uint64) for _ in range(4)]
    recv_counts = np.ascontiguousarray(recv_counts, np.uint64)
    recv_offsets = np.ascontiguousarray(recv_offsets, np.uint64)
    rc = ref().ref_lcp_merge(_p(chars), chars.size, _p(lcps), n, p, _p(recv_counts), _p(recv_offsets),
                             *(_p(x) for x in o))
    assert rc == 0, rc
    return tuple(x[:n] for x in o)


# ------------------------------------------------------------------ Golomb ----
def _golomb_lib():
    L = lib()
    if not hasattr(L, "_golomb_set"):
        L.oracle_golomb_param.restype = _U64
        L.oracle_golomb_param.argtypes = [_U64, _U64]
        L.oracle_golomb_param_hashes.restype = _U64
        L.oracle_golomb_param_hashes.argtypes = [_U64, _U32]
        L.oracle_golomb_encode.restype = ctypes.c_int64
        L.oracle_golomb_encode.argtypes = [_P, _P, _U32, _P, _P, _U64, _P]
        L.oracle_golomb_decode.restype = ctypes.c_int64
        L.oracle_golomb_decode.argtypes = [_P, _U64, _P, _U64, _P, _U32, ctypes.POINTER(_U32)]
        L._golomb_set = True
    return L


def golomb_param(max_value: int, count: int) -> int:
    """getB (golomb_encoding.hpp:50-59)."""
    return int(_golomb_lib().oracle_golomb_param(max_value, count))


def golomb_param_hashes(count: int, p: int) -> int:
    """b of the hash exchange to one of p PEs that receives count hashes."""
    return int(_golomb_lib().oracle_golomb_param_hashes(count, p))


def golomb_encode(values, counts, bs):
    """Golomb/delta blocks of sorted ranges (the hash exchange's format):
    returns (words u64, words per range)."""
    v = np.ascontiguousarray(values, dtype=np.uint64)
    c = np.ascontiguousarray(counts, dtype=np.uint64)
    b = np.ascontiguousarray(bs, dtype=np.uint64)
    cap = int(3 * len(c) + 2 * len(v) + 8 + sum(int(x) for x in golomb_unary_words(v, c, b)))
    out = np.zeros(cap, np.uint64)
    rw = np.zeros(len(c), np.uint64)
    n = _golomb_lib().oracle_golomb_encode(v.ctypes.data, c.ctypes.data, len(c), b.ctypes.data, out.ctypes.data,
                                           cap, rw.ctypes.data)
    if n < 0:
        raise RuntimeError("golomb_encode: output larger than planned")
    return out[:n], rw


def golomb_unary_words(v, c, b):
    """Upper bound of the words the unary parts of each range take."""
    off = 0
    for cnt, bb in zip(c.tolist(), b.tolist()):
        seg = v[off:off + cnt]
        off += cnt
        yield 0 if cnt < 2 else int(((seg[-1] - seg[0]) // np.uint64(bb))) // 64 + 2


def golomb_decode(words, max_blocks=1 << 20, cap=None):
    """Values and per-block counts of back-to-back blocks."""
    w = np.ascontiguousarray(words, dtype=np.uint64)
    cap = cap if cap is not None else int(64 * len(w) + 8)
    out = np.zeros(max(cap, 1), np.uint64)
    bc = np.zeros(max_blocks, np.uint64)
    nb = _U32(0)
    n = _golomb_lib().oracle_golomb_decode(w.ctypes.data, len(w), out.ctypes.data, cap, bc.ctypes.data, max_blocks,
                                           ctypes.byref(nb))
    if n < 0:
        raise ValueError("golomb_decode: malformed block")
    return out[:n], bc[:nb.value]


def ref_golomb_block(values, b):
    """The reference's own coder (compiled from src/encoding/golomb_encoding.hpp)
    on one block, framed as AllToAllHashesGolomb frames it."""
    v = np.ascontiguousarray(values, dtype=np.uint64)
    cap = int(3 + 2 * len(v) + 8 + (int((v[-1] - v[0]) // np.uint64(b)) // 64 + 2 if len(v) > 1 else 0))
    out = np.zeros(cap, np.uint64)
    n = ref().ref_golomb_block(v.ctypes.data, len(v), b, out.ctypes.data, cap)
    if n < 0:
        raise RuntimeError("ref_golomb_block: output larger than planned")
    return out[:n]


def ref_golomb_unblock(words, cap):
    w = np.ascontiguousarray(words, dtype=np.uint64)
    out = np.zeros(max(cap, 1), np.uint64)
    n = ref().ref_golomb_unblock(w.ctypes.data, len(w), out.ctypes.data, cap)
    if n < 0:
        raise RuntimeError("ref_golomb_unblock failed")
    return out[:n]

