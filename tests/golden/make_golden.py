"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a container where the reference tree is mounted and oracle/_ref is
built (`make -C oracle`):  python tests/golden/make_golden.py

Fixtures (JSON, small):
  xxh64_ref.json        XXH64 (seed 0) of seeded byte strings of every length
                        0..130 and some up to 600, from the reference's
                        hash/xxhash.hpp (xxh::hash_state_t<64>).
  dp_ref.json           the reference's radixsort_CI3 + computeDistinguishingPrefixes
                        (one PE, via oracle/_ref/libref_dp.so) on seeded sets:
                        input strings, sorted order, LCPs, DP lengths.
  merge_ref.json        the reference's LcpStringLoserTree_ on receive containers
                        (prefix-compressed strings as the PD exchange delivers them).
  pd_exchange_kat.json  the PD exchange known-answer test of
                        src/tests/alltoallStrings_tests.cpp:129-163 restated:
                        per simulated PE count, the sender-side strings, LCPs,
                        DP lengths and send counts, and the expected receive
                        bytes and LCPs of getExpectedRawStringsForPrefixDoubling
                        (:62-72), ..._Duplicates... (:74-84), getExpectedLcpValues (:86-93).
  golomb_ref.json       the reference's Golomb/delta coder (getDeltaEncoding of
                        src/encoding/golomb_encoding.hpp over thrill's bit
                        streams, via oracle/_ref/libref.so) on seeded sorted
                        blocks, framed [S, b, ...] as AllToAllHashesGolomb
                        frames them, and getB on a few (max, count) pairs.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from inputs import long_prefix, random_strings, with_duplicates  # noqa: E402


def hexs(strs):
    return [s.hex() for s in strs]


def make_xxh():
    rng = np.random.default_rng(11)
    vecs = []
    lens = list(range(0, 131)) + [192, 255, 256, 257, 300, 511, 512, 520, 600]
    for L in lens:
        data = bytes(rng.integers(0, 256, size=L).astype(np.uint8))
        vecs.append({"data": data.hex(), "xxh64": format(oracle.ref_xxh64(data), "016x")})
    vecs.append({"data": b"HELLOWOR".hex(), "xxh64": format(oracle.ref_xxh64(b"HELLOWOR"), "016x")})
    return vecs


def dp_sets():
    return {
        "binary": random_strings(600, 0, 30, b"AB", 21),
        "dups": with_duplicates(random_strings(500, 0, 20, b"ACGT", 22)),
        "long_prefix": long_prefix(300, 300, 30, 23),
        "dn_rule": [b"A" * 45 + bytes([65 + (i // 26 ** k) % 26 for k in (4, 3, 2, 1, 0)]) +
                    bytes(np.random.default_rng(i).integers(65, 91, 50).astype(np.uint8)) for i in range(400)],
    }


def make_dp():
    out = {}
    for name, strs in dp_sets().items():
        order, lcp, dp = oracle.ref_dp_single_pe(strs)
        out[name] = {"strings": hexs(strs), "order": order.tolist(), "lcp": lcp.tolist(), "dp": dp.tolist()}
    return out


def make_merge():
    out = {}
    for name, strs, p in [("binary_p4", random_strings(800, 0, 24, b"AB", 31), 4),
                          ("dups_p3", with_duplicates(random_strings(600, 0, 12, b"ACG", 32), 0.5), 3),
                          ("prefix_p5", long_prefix(500, 40, 6, 33), 5)]:
        s = oracle.Strings(*_arena(strs))
        pb = np.array([q * len(strs) // p for q in range(p + 1)], np.uint64)
        order, lcp = oracle.local_sort(s, pb)
        dp, _ = oracle.dp_rounds(s, pb, order, lcp)
        iv = oracle.partition(s, pb, order, dp)
        ex = oracle.exchange(s, pb, order, lcp, dp, iv)
        pes = []
        start = 0
        for r in range(p):
            cnt = int(ex["counts"][r].sum())
            cb, ce = int(ex["char_begin"][r]), int(ex["char_begin"][r + 1])
            lcps = ex["lcp"][start:start + cnt]
            idx, pe, mlcp, old = oracle.ref_lcp_merge(ex["chars"][cb:ce], lcps, ex["counts"][r], ex["offsets"][r])
            pes.append({"chars": ex["chars"][cb:ce].tobytes().hex(), "lcp": lcps.tolist(),
                        "counts": ex["counts"][r].tolist(), "offsets": ex["offsets"][r].tolist(),
                        "index": idx.tolist(), "pe": pe.tolist(), "merged_lcp": mlcp.tolist(), "old_lcp": old.tolist()})
            start += cnt
        out[name] = {"p": p, "pes": pes}
    return out


def _arena(strs):
    lens = np.array([len(x) for x in strs], np.uint32)
    offs = np.zeros(len(strs), np.uint64)
    if len(strs):
        offs[1:] = np.cumsum(lens.astype(np.uint64) + 1)[:-1]
    chars = np.frombuffer(b"".join(x + b"\0" for x in strs) + b"\0" * 32, np.uint8).copy()
    return chars, offs, lens


def make_kat():
    """alltoallStrings_tests.cpp:129-163 for p = 1, 2, 4, 8 simulated PEs."""
    common, suffix, per = 10, 20, 5
    cases = []
    for p in (1, 2, 4, 8):
        for dup in (False, True):
            pes = []
            for rank in range(p):
                # generateRawStrings (:17-33): p blocks of `per` strings
                strs = []
                for _ in range(p):
                    for i in range(1, per + 1):
                        strs.append(bytes([rank + 1]) * common + bytes([i]) + bytes([rank + 1]) * suffix)
                lcps = [common] * (per * p)
                lcps[0] = 0
                dpl = common if dup else common + 1
                pes.append({"strings": hexs(strs), "lcp": lcps, "dp": [dpl] * (per * p), "send": [per] * p})
            exp_raw, exp_lcp = [], []
            for pe in range(p):
                raw = bytes([pe + 1]) * common
                if dup:
                    raw += b"\0" * per  # getExpectedRawStrings_DuplicatesForPrefixDoubling (:74-84)
                else:
                    raw += b"".join(bytes([i + 1, 0]) for i in range(per))  # (:62-72)
                exp_raw.append(raw)
                exp_lcp += [0] + [common] * (per - 1)  # getExpectedLcpValues (:86-93)
            cases.append({"p": p, "simulate_duplicates": dup, "pes": pes,
                          "expected_raw": b"".join(exp_raw).hex(), "expected_lcp": exp_lcp})
    return cases


def golomb_blocks():
    rng = np.random.default_rng(2024)
    cases = []
    for k in range(24):
        c = int(rng.integers(1, 120))
        kind = k % 4
        if kind == 0:  # hashes: the 64-bit range
            v = np.sort(rng.integers(0, 2**64 - 1, c, dtype=np.uint64))
            b = int(oracle.golomb_param_hashes(c, 4))
        elif kind == 1:  # duplicate positions plus an offset: b >= 8
            v = np.sort(rng.choice(5000, c, replace=False)).astype(np.uint64) + np.uint64(123456)
            b = max(8, oracle.golomb_param(5000, c))
        elif kind == 2:  # small gaps, b not a power of two
            v = np.cumsum(rng.integers(0, 40, c)).astype(np.uint64)
            b = [3, 5, 7, 1000, 20000000000][k % 5]
        else:  # a gap that needs more than 64 unary bits
            v = np.cumsum(rng.integers(0, 3, c)).astype(np.uint64)
            v[c // 2:] += np.uint64(100000)
            b = 8
        cases.append((v, b))
    return cases


def make_golomb():
    blocks = []
    for v, b in golomb_blocks():
        w = oracle.ref_golomb_block(v, b)
        blocks.append({"values": [str(x) for x in v.tolist()], "b": int(b), "words": [str(x) for x in w.tolist()]})
    params = [[str(m), str(c), str(int(oracle.ref().ref_golomb_param(m, c)))]
              for m, c in [(2**64 - 1, 1), (2**64 - 1, 3), ((2**64 - 1) // 4, 1000), (100, 7), (7, 100),
                           (2**63, 2**62 + 1), (10**12, 999), (0, 5), (5, 0)]]
    return {"blocks": blocks, "params": params}


def main():
    if not oracle.ref_available() or not oracle.ref_dp_available():
        sys.exit("oracle/_ref is not built: run `make -C oracle` where the reference tree is present")
    with open(os.path.join(HERE, "xxh64_ref.json"), "w") as f:
        json.dump(make_xxh(), f)
    with open(os.path.join(HERE, "dp_ref.json"), "w") as f:
        json.dump(make_dp(), f)
    with open(os.path.join(HERE, "merge_ref.json"), "w") as f:
        json.dump(make_merge(), f)
    with open(os.path.join(HERE, "pd_exchange_kat.json"), "w") as f:
        json.dump(make_kat(), f)
    with open(os.path.join(HERE, "golomb_ref.json"), "w") as f:
        json.dump(make_golomb(), f)


if __name__ == "__main__":
    main()
