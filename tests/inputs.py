"""Seeded test inputs shared by the CPU and GPU tests (all small enough for the oracle)."""
import numpy as np


def random_strings(n, min_len, max_len, alphabet=b"AB", seed=0):
    rng = np.random.default_rng(seed)
    al = np.frombuffer(alphabet, dtype=np.uint8)
    lens = rng.integers(min_len, max_len + 1, size=n)
    return [al[rng.integers(0, len(al), size=int(L))].tobytes() for L in lens]


def with_duplicates(strs, frac=0.3, seed=1):
    rng = np.random.default_rng(seed)
    out = list(strs)
    for i in range(len(out)):
        if rng.random() < frac:
            out[i] = out[int(rng.integers(0, len(out)))]
    return out


def long_prefix(n, prefix_len, tail, seed=2):
    rng = np.random.default_rng(seed)
    pre = b"A" * prefix_len
    return [pre + bytes(rng.integers(65, 91, size=int(rng.integers(0, tail + 1))).astype(np.uint8))
            for _ in range(n)]


def prefixes_of_each_other(n, seed=3):
    rng = np.random.default_rng(seed)
    base = bytes(rng.integers(65, 69, size=300).astype(np.uint8))
    return [base[:int(rng.integers(0, 301))] for _ in range(n)]


def shared_head(n, head_len=300, tail=20, seed=8):
    """Strings that copy a random length of one shared head, then random tail
    bytes: a chain of nested groups that each lose a few strings per byte."""
    rng = np.random.default_rng(seed)
    head = bytes(rng.integers(65, 91, size=head_len).astype(np.uint8))
    out = []
    for _ in range(n):
        k = int(rng.integers(0, head_len + 1))
        out.append(head[:k] + bytes(rng.integers(65, 91, size=int(rng.integers(0, tail + 1))).astype(np.uint8)))
    return out


def run_suffixes(seed=9, max_len=256):
    """All suffixes (truncated) of a text with long single-letter and periodic
    runs: suffixes inside a run share prefixes that end one byte apart."""
    rng = np.random.default_rng(seed)
    parts = []
    for _ in range(12):
        r = int(rng.integers(0, 3))
        if r == 0:
            parts.append(b"A" * int(rng.integers(100, 700)))
        elif r == 1:
            parts.append(b"CG" * int(rng.integers(50, 300)))
        else:
            parts.append(bytes(rng.integers(65, 69, size=int(rng.integers(5, 60))).astype(np.uint8)))
    text = b"".join(parts)
    return [text[i:i + max_len] for i in range(len(text))]


def cases():
    """(name, list of byte strings) covering the edge cases the reference's tests touch."""
    return [
        ("empty", []),
        ("single", [b"HELLO"]),
        ("single_empty", [b""]),
        ("two_equal", [b"ABC", b"ABC"]),
        ("all_identical", [b"ABCDEFGHIJKLMNOPQRSTUVWXYZ"] * 50),
        ("empty_strings", [b""] * 5 + [b"A", b"", b"B"]),
        ("binary_alphabet", random_strings(3000, 0, 40, b"AB", 4)),
        ("dups", with_duplicates(random_strings(2000, 0, 30, b"ACGT", 5))),
        ("long_prefix", long_prefix(1500, 600, 40)),
        ("prefix_chain", prefixes_of_each_other(800)),
        ("long_strings", random_strings(400, 900, 2100, b"AB", 6)),
        ("wide_alphabet", random_strings(2000, 1, 64, bytes(range(1, 256)), 7)),
        ("shared_head", shared_head(3000)),
        ("run_suffixes", run_suffixes()),
    ]
