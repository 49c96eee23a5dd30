"""dsss_b200 — Python front-end over libdsss (the C ABI in include/dsss.h).

Every call goes through the shared library with ctypes; torch is used only for
device memory and streams.  Importing fails loudly when libdsss.so is missing:
there is no CPU fallback for any entry point.

The directory name is not a Python identifier; load it with ``load_package()``
from ``__graft_entry__`` (which registers it as ``dsss_b200``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdsss.so")

DSSS_OK = 0
ERRORS = {-22: "EINVAL", -12: "ENOMEM", -110: "ETIMEDOUT", -5: "EDEVICE", -95: "ENOTSUP"}
SAMPLER_NUM_STRINGS = 0
SAMPLER_INDEXED_NUM_STRINGS = 2
FLAG_LOCAL_LCP = 1
PAD = 64  # bytes of zero padding behind device arenas (the ABI asks for >= 32)


class DsssError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Arena(ctypes.Structure):
    _fields_ = [("chars", ctypes.c_void_p), ("char_bytes", ctypes.c_uint64), ("offsets", ctypes.c_void_p),
                ("lengths", ctypes.c_void_p), ("n", ctypes.c_uint64)]


class Opts(ctypes.Structure):
    _fields_ = [("sampler", ctypes.c_uint32), ("sampling_factor", ctypes.c_uint32),
                ("small_sort_max", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


class PdResult(ctypes.Structure):
    _fields_ = [("local_order", ctypes.c_void_p), ("local_lcp", ctypes.c_void_p), ("dp", ctypes.c_void_p),
                ("intervals", ctypes.c_void_p), ("perm_index", ctypes.c_void_p), ("perm_pe", ctypes.c_void_p),
                ("merged_lcp", ctypes.c_void_p), ("recv_counts", ctypes.c_void_p)]


class MsResult(ctypes.Structure):
    _fields_ = [("local_order", ctypes.c_void_p), ("intervals", ctypes.c_void_p), ("chars", ctypes.c_void_p),
                ("chars_capacity", ctypes.c_uint64), ("offsets", ctypes.c_void_p), ("lengths", ctypes.c_void_p),
                ("lcp", ctypes.c_void_p), ("source", ctypes.c_void_p), ("recv_counts", ctypes.c_void_p),
                ("avg_lcp", ctypes.c_uint64)]


class HqResult(ctypes.Structure):
    _fields_ = [("counts", ctypes.c_void_p), ("chars", ctypes.c_void_p), ("chars_capacity", ctypes.c_uint64),
                ("offsets", ctypes.c_void_p), ("lengths", ctypes.c_void_p), ("source", ctypes.c_void_p),
                ("levels", ctypes.c_uint32)]


class Tuning(ctypes.Structure):
    _fields_ = [("sort_small_max", ctypes.c_int64), ("sort_pivot", ctypes.c_int64), ("dp_filter_min", ctypes.c_int64),
                ("best_ms", ctypes.c_double), ("default_ms", ctypes.c_double), ("settings_tried", ctypes.c_uint32),
                ("sort_split_min", ctypes.c_int64), ("sort_bits", ctypes.c_int64),
                ("sort_seg_bits", ctypes.c_int64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workers", ctypes.c_uint32), ("p", ctypes.c_uint32),
                ("max_sets", ctypes.c_uint32), ("max_batch_strings", ctypes.c_uint64),
                ("hbm_budget", ctypes.c_uint64), ("opts", Opts), ("flags", ctypes.c_uint32),
                ("reserve_bytes", ctypes.c_uint64)]


class RequestStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("batch_sets", ctypes.c_uint32), ("batch_id", ctypes.c_uint64),
                ("batch_strings", ctypes.c_uint64), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("t_copied", ctypes.c_double), ("t_sorted", ctypes.c_double),
                ("error", ctypes.c_char * 160)]


class ServerInfo(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_uint64), ("reserved_bytes", ctypes.c_uint64),
                ("max_reserved_bytes", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("batched_requests", ctypes.c_uint64), ("hbm_budget", ctypes.c_uint64)]


_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_I = ctypes.c_int
_SIGS = {
    "dsss_ctx_create": (_I, [_I, _U64, ctypes.POINTER(_P)]),
    "dsss_ctx_destroy": (_I, [_P]),
    "dsss_ctx_scratch_bytes": (_U64, [_P]),
    "dsss_last_error": (ctypes.c_char_p, []),
    "dsss_ctx_set_timing": (_I, [_P, _I]),
    "dsss_ctx_kernel_times": (_I, [_P, ctypes.c_char_p, _U64]),
    "dsss_abi_version": (_I, []),
    "dsss_pd_sort": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, ctypes.POINTER(Opts), ctypes.POINTER(PdResult), _P]),
    "dsss_ms_sort": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, ctypes.POINTER(Opts), ctypes.POINTER(MsResult), _P]),
    "dsss_hq_sort": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _U64, ctypes.POINTER(HqResult), _P]),
    "dsss_distribute_lines": (_I, [_P, _P, _U64, _U64, _U32, _P, _U64, _P, _P, _U64, _P, _P, _P, _P]),
    "dsss_varint_encode": (_I, [_P, _P, _U64, _P, _U32, _P, _U64, _P, _P, _P]),
    "dsss_varint_decode": (_I, [_P, _P, _U64, _P, _U64, _P]),
    "dsss_golomb_param": (_U64, [_U64, _U64]),
    "dsss_golomb_param_hashes": (_U64, [_U64, _U32]),
    "dsss_golomb_encode": (_I, [_P, _P, _P, _U32, _P, _P, _U64, ctypes.POINTER(_U64), _P, _P]),
    "dsss_golomb_decode": (_I, [_P, _P, _U64, _P, _U64, ctypes.POINTER(_U64), _P, _U32, ctypes.POINTER(_U32), _P]),
    "dsss_pd_sort_host": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, ctypes.POINTER(Opts), ctypes.POINTER(PdResult),
                               _P]),
    "dsss_pd_sort_batched": (_I, [_P, ctypes.POINTER(Arena), _U32, _U32, _P, ctypes.POINTER(Opts),
                                  ctypes.POINTER(PdResult), _P]),
    "dsss_pd_sort_batched_host": (_I, [_P, ctypes.POINTER(Arena), _U32, _U32, _P, ctypes.POINTER(Opts),
                                       ctypes.POINTER(PdResult), _P]),
    "dsss_clock_now": (ctypes.c_double, []),
    "dsss_dp_classify_hash": (_I, [_P, ctypes.POINTER(Arena), _P, _P, _P, _U32, _P, _P, _P, _P, ctypes.POINTER(_U64),
                                   _P]),
    "dsss_hash_route": (_I, [_P, _P, _P, _U64, _U32, _P, _P, _P, _P]),
    "dsss_hash_dups": (_I, [_P, _P, _U64, _P, _P]),
    "dsss_hash_sort": (_I, [_P, _P, _P, _U64, _P, _P, _P]),
    "dsss_dp_apply": (_I, [_P, _P, _P, _U64, _P, _U64, ctypes.POINTER(_U64), _P]),
    "dsss_pack_strings": (_I, [_P, ctypes.POINTER(Arena), _P, _P, _U64, _P, _U64, _P, _P, ctypes.POINTER(_U64), _P]),
    "dsss_partition_search": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _P, ctypes.POINTER(Arena), _P, _U32, _P, _I,
                                   _P, _P]),
    "dsss_bucket_send": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _P, _P, _P, _U32, _U32, _P, _P, _U64,
                              ctypes.POINTER(_U64), _P, _P, _P, _P, _P, _P]),
    "dsss_regroup": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, _U64, _P]),
    "dsss_tune_set": (_I, [ctypes.c_char_p, ctypes.c_int64]),
    "dsss_tune_get": (_I, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
    "dsss_autotune": (_I, [_P, ctypes.POINTER(Arena), _U32, _U32, _P, ctypes.POINTER(Opts), _U32, ctypes.POINTER(Tuning),
                           _P]),
    "dsss_server_create": (_I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    "dsss_server_submit": (_I, [_P, ctypes.POINTER(Arena), _P, ctypes.POINTER(PdResult), ctypes.POINTER(_U64)]),
    "dsss_server_wait": (_I, [_P, _U64, ctypes.c_int64, ctypes.POINTER(RequestStats)]),
    "dsss_server_info": (_I, [_P, ctypes.POINTER(ServerInfo)]),
    "dsss_server_footprint": (_U64, [_P, _U64, _U64]),
    "dsss_server_destroy": (_I, [_P]),
    "dsss_local_sort_lcp": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, ctypes.POINTER(Opts), _P, _P, _P]),
    "dsss_dp_prefixes": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _P, _P, _P, _P, _U32, _P, _P]),
    "dsss_prefix_hash": (_I, [ctypes.POINTER(Arena), _P, _U64, _U32, _P, _P]),
    "dsss_dp_round": (_I, [_P, ctypes.POINTER(Arena), _P, _P, _P, _U64, _U32, _P, _P, _P, _P]),
    "dsss_bucket_scatter": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _P, _P, _P, _P, _P, _U64, _P, _P, _P, _P, _P,
                                 _P, _P, _P, _P]),
    "dsss_lcp_merge": (_I, [_P, _P, _U64, _P, _P, _U64, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "dsss_lcp_merge_strings": (_I, [_P, _P, _U64, _P, _P, _U64, _U32, _U32, _P, _P, _P, _P, _P, _U64, _P, _P, _P,
                                    _P]),
    "dsss_partition": (_I, [_P, ctypes.POINTER(Arena), _U32, _P, _P, _P, ctypes.POINTER(Opts), _P, _P]),
    "dsss_adjacent_lcp": (_I, [_P, ctypes.POINTER(Arena), _P, _U64, _P, _P]),
    "dsss_adjacent_lcp_noalloc": (_I, [ctypes.POINTER(Arena), _P, _U64, _P, _P]),
    "dsss_gen_dn": (_I, [_U64, _U32, _U32, _U32, _U32, ctypes.c_double, _U64, _P, _P, _P, _P]),
    "dsss_gen_markov_text": (_I, [_U64, ctypes.c_double, _U64, _P]),
    "dsss_gen_suffixes": (_I, [_U64, _U32, _P, _P]),
    "dsss_gen_request": (_I, [_U64, _U32, _U32, ctypes.c_double, _U64, _P, _P, _P, _P]),
    "dsss_gen_dn_dev": (_I, [_P, _U64, _U32, _U32, _U32, _U32, ctypes.c_double, _U64, _P, _P, _P, _P, _P]),
    "dsss_gen_suffixes_dev": (_I, [_U64, _U32, _P, _P, _P]),
    "dsss_gen_request_dev": (_I, [_P, _U64, _U32, _U32, ctypes.c_double, _U64, _P, _P, _P, _P, _P]),
}

_lib = None


def lib():
    """The loaded libdsss (raises if the library was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run build() (python build.py) first")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc: int):
    if rc != DSSS_OK:
        raise DsssError(rc, lib().dsss_last_error().decode(errors="replace"))


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


# ------------------------------------------------------------------ inputs --
@dataclass
class HostStrings:
    """Strings in host memory: chars (uint8, padded), offsets (uint64), lengths (uint32)."""
    chars: np.ndarray
    offsets: np.ndarray
    lengths: np.ndarray
    char_bytes: int

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0])

    def get(self, i: int) -> bytes:
        o, l = int(self.offsets[i]), int(self.lengths[i])
        return self.chars[o:o + l].tobytes()

    def arena(self) -> Arena:
        return Arena(_ptr(self.chars), self.char_bytes, _ptr(self.offsets), _ptr(self.lengths), self.n)


def _alloc_host(nbytes: int, dtype, pinned: bool):
    if pinned:
        import torch
        t = torch.empty(nbytes // np.dtype(dtype).itemsize, dtype=_TORCH_DT[np.dtype(dtype)], pin_memory=True)
        return t.numpy()
    return np.empty(nbytes // np.dtype(dtype).itemsize, dtype=dtype)


def _torch_dt():
    import torch
    return {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint32): torch.uint32, np.dtype(np.uint64): torch.uint64}


class _LazyDT(dict):
    def __missing__(self, k):
        self.update(_torch_dt())
        return dict.__getitem__(self, k)


_TORCH_DT = _LazyDT()


def gen_dn(n: int, length: int, k: int, seed: int = 1, long_len: int = 0, long_k: int = 0, frac_long: float = 0.0,
           pinned: bool = False) -> HostStrings:
    """D/N-ratio strings (see dsss_gen_dn); each string is followed by a NUL."""
    cb = ctypes.c_uint64(0)
    check(lib().dsss_gen_dn(n, length, k, long_len, long_k, frac_long, seed, None, None, None, ctypes.byref(cb)))
    total = cb.value
    chars = _alloc_host(total + PAD, np.uint8, pinned)
    offs = _alloc_host(max(n, 1) * 8, np.uint64, pinned)[:n]
    lens = _alloc_host(max(n, 1) * 4, np.uint32, pinned)[:n]
    check(lib().dsss_gen_dn(n, length, k, long_len, long_k, frac_long, seed, _ptr(chars), _ptr(offs), _ptr(lens),
                            ctypes.byref(cb)))
    chars[total:] = 0
    return HostStrings(chars, offs, lens, total)


def gen_suffix_strings(text_len: int, max_len: int = 256, seed: int = 1, copy_prob: float = 0.01,
                       pinned: bool = False) -> HostStrings:
    """All suffixes of a seeded order-3 Markov ACGT text, truncated to max_len."""
    chars = _alloc_host(text_len + PAD, np.uint8, pinned)
    check(lib().dsss_gen_markov_text(text_len, copy_prob, seed, _ptr(chars)))
    chars[text_len:] = 0
    offs = _alloc_host(max(text_len, 1) * 8, np.uint64, pinned)[:text_len]
    lens = _alloc_host(max(text_len, 1) * 4, np.uint32, pinned)[:text_len]
    check(lib().dsss_gen_suffixes(text_len, max_len, _ptr(offs), _ptr(lens)))
    return HostStrings(chars, offs, lens, text_len)


def gen_request(n: int, seed: int, min_len: int = 8, max_len: int = 256, zipf_s: float = 1.2,
                pinned: bool = False) -> HostStrings:
    cb = ctypes.c_uint64(0)
    check(lib().dsss_gen_request(n, min_len, max_len, zipf_s, seed, None, None, None, ctypes.byref(cb)))
    total = cb.value
    chars = _alloc_host(total + PAD, np.uint8, pinned)
    offs = _alloc_host(max(n, 1) * 8, np.uint64, pinned)[:n]
    lens = _alloc_host(max(n, 1) * 4, np.uint32, pinned)[:n]
    check(lib().dsss_gen_request(n, min_len, max_len, zipf_s, seed, _ptr(chars), _ptr(offs), _ptr(lens),
                                 ctypes.byref(cb)))
    chars[total:] = 0
    return HostStrings(chars, offs, lens, total)


def gen_dn_device(ctx, n: int, length: int, k: int, seed: int = 1, long_len: int = 0, long_k: int = 0,
                  frac_long: float = 0.0, stream=None) -> "DeviceStrings":
    """gen_dn generated in device memory (dsss_gen_dn_dev): the same bytes,
    no host round trip."""
    import torch
    dev = f"cuda:{ctx.device}"
    cb = ctypes.c_uint64(0)
    check(lib().dsss_gen_dn_dev(ctx.h, n, length, k, long_len, long_k, frac_long, seed, None, None, None,
                                ctypes.byref(cb), _stream_ptr(stream)))
    total = cb.value
    chars = torch.zeros(total + PAD, dtype=torch.uint8, device=dev)
    offs = torch.empty(max(n, 1), dtype=torch.int64, device=dev)[:n]
    lens = torch.empty(max(n, 1), dtype=torch.int32, device=dev)[:n]
    check(lib().dsss_gen_dn_dev(ctx.h, n, length, k, long_len, long_k, frac_long, seed, chars.data_ptr(),
                                offs.data_ptr(), lens.data_ptr(), ctypes.byref(cb), _stream_ptr(stream)))
    return DeviceStrings(None, chars=chars, offsets=offs, lengths=lens, char_bytes=total)


def gen_request_device(ctx, n: int, seed: int, min_len: int = 8, max_len: int = 256, zipf_s: float = 1.2,
                       stream=None) -> "DeviceStrings":
    """gen_request generated in device memory (dsss_gen_request_dev)."""
    import torch
    dev = f"cuda:{ctx.device}"
    cb = ctypes.c_uint64(0)
    check(lib().dsss_gen_request_dev(ctx.h, n, min_len, max_len, zipf_s, seed, None, None, None, ctypes.byref(cb),
                                     _stream_ptr(stream)))
    total = cb.value
    chars = torch.zeros(total + PAD, dtype=torch.uint8, device=dev)
    offs = torch.empty(max(n, 1), dtype=torch.int64, device=dev)[:n]
    lens = torch.empty(max(n, 1), dtype=torch.int32, device=dev)[:n]
    check(lib().dsss_gen_request_dev(ctx.h, n, min_len, max_len, zipf_s, seed, chars.data_ptr(), offs.data_ptr(),
                                     lens.data_ptr(), ctypes.byref(cb), _stream_ptr(stream)))
    return DeviceStrings(None, chars=chars, offsets=offs, lengths=lens, char_bytes=total)


def gen_suffix_strings_device(text_len: int, max_len: int = 256, seed: int = 1, copy_prob: float = 0.01,
                              device="cuda", stream=None) -> "DeviceStrings":
    """gen_suffix_strings with the suffix views made on the device
    (dsss_gen_suffixes_dev); only the text (text_len bytes) is made on the
    host and copied in."""
    import torch
    text = np.zeros(text_len + PAD, np.uint8)
    check(lib().dsss_gen_markov_text(text_len, copy_prob, seed, _ptr(text)))
    chars = torch.from_numpy(text).to(device)
    offs = torch.empty(max(text_len, 1), dtype=torch.int64, device=device)[:text_len]
    lens = torch.empty(max(text_len, 1), dtype=torch.int32, device=device)[:text_len]
    check(lib().dsss_gen_suffixes_dev(text_len, max_len, offs.data_ptr(), lens.data_ptr(), _stream_ptr(stream)))
    return DeviceStrings(None, chars=chars, offsets=offs, lengths=lens, char_bytes=text_len)


def from_bytes_list(strs) -> HostStrings:
    """Arena of Python byte strings laid out back to back with NULs."""
    n = len(strs)
    lens = np.array([len(s) for s in strs], dtype=np.uint32)
    offs = np.zeros(n, dtype=np.uint64)
    if n:
        offs[1:] = np.cumsum(lens.astype(np.uint64) + 1)[:-1]
    total = int(lens.astype(np.uint64).sum()) + n
    chars = np.zeros(total + PAD, dtype=np.uint8)
    for i, s in enumerate(strs):
        o = int(offs[i])
        chars[o:o + len(s)] = np.frombuffer(s, dtype=np.uint8)
    return HostStrings(chars, offs, lens, total)


def equal_parts(n: int, p: int) -> np.ndarray:
    """PE boundaries of p contiguous slices with equal string counts."""
    return np.array([q * n // p for q in range(p + 1)], dtype=np.uint64)


def concat_sets(sets, pinned: bool = False):
    """One arena holding several string sets back to back; returns it and the
    set bounds (len(sets) + 1 string ids)."""
    n = sum(h.n for h in sets)
    total = sum(h.char_bytes for h in sets)
    chars = _alloc_host(total + PAD, np.uint8, pinned)
    offs = _alloc_host(max(n, 1) * 8, np.uint64, pinned)[:n]
    lens = _alloc_host(max(n, 1) * 4, np.uint32, pinned)[:n]
    set_begin = np.zeros(len(sets) + 1, dtype=np.uint64)
    cpos, spos = 0, 0
    for k, h in enumerate(sets):
        chars[cpos:cpos + h.char_bytes] = h.chars[:h.char_bytes]
        offs[spos:spos + h.n] = h.offsets + np.uint64(cpos)
        lens[spos:spos + h.n] = h.lengths
        cpos += h.char_bytes
        spos += h.n
        set_begin[k + 1] = spos
    chars[total:] = 0
    return HostStrings(chars, offs, lens, total), set_begin


def batched_parts(set_begin, p: int) -> np.ndarray:
    """PE boundaries (nsets*p + 1) of p equal slices inside every set."""
    sb = np.asarray(set_begin, dtype=np.uint64)
    out = [0]
    for s in range(len(sb) - 1):
        n = int(sb[s + 1] - sb[s])
        out.extend(int(sb[s]) + q * n // p for q in range(1, p + 1))
    return np.array(out, dtype=np.uint64)


# ------------------------------------------------------------------ device --
class DeviceStrings:
    """A device copy of HostStrings (torch tensors; chars padded with zeros),
    or device tensors made by the device-side generators (hs=None)."""

    def __init__(self, hs: Optional[HostStrings], device="cuda", chars=None, offsets=None, lengths=None,
                 char_bytes=0):
        import torch
        if hs is None:
            self.chars, self.offsets, self.lengths = chars, offsets, lengths
            self.char_bytes = int(char_bytes)
            self.n = int(offsets.numel())
            return
        self.chars = torch.from_numpy(hs.chars).to(device)
        self.offsets = torch.from_numpy(hs.offsets.view(np.int64)).to(device)
        self.lengths = torch.from_numpy(hs.lengths.view(np.int32)).to(device)
        self.char_bytes = hs.char_bytes
        self.n = hs.n

    def arena(self) -> Arena:
        return Arena(self.chars.data_ptr(), self.char_bytes, self.offsets.data_ptr(), self.lengths.data_ptr(), self.n)


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Context:
    """Owns the library's reusable device scratch (one per host thread)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = ctypes.c_void_p()
        check(lib().dsss_ctx_create(device, hbm_budget, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().dsss_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def scratch_bytes(self) -> int:
        return int(lib().dsss_ctx_scratch_bytes(self.h))

    def set_timing(self, on: bool):
        """Per-kernel CUDA-event timing of every launch this context makes."""
        check(lib().dsss_ctx_set_timing(self.h, 1 if on else 0))

    def kernel_times(self) -> dict:
        """{kernel: (launches, total_ms)} for the launches timed since set_timing(True)."""
        buf = ctypes.create_string_buffer(1 << 16)
        check(lib().dsss_ctx_kernel_times(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, k, ms = line.split()
            out[name] = (int(k), float(ms))
        return out


def _opts(sampler=0, sampling_factor=2, small_sort_max=0, flags=0) -> Opts:
    return Opts(sampler, sampling_factor, small_sort_max, flags)


def _empty(n, dtype="int32", device="cuda"):
    import torch
    return torch.empty(max(n, 1), dtype=getattr(torch, dtype), device=device)


def pd_sort(ctx: Context, ds: DeviceStrings, p: int, part_begin=None, sampler: int = 0, merged_lcp: bool = True,
            local_lcp: bool = False, small_sort_max: int = 0, stream=None, out=None):
    """DistributedPrefixDoublingSort::sort on the device.  Returns a dict of
    torch tensors (device) plus host numpy intervals / recv_counts."""
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    if out is None:
        out = dict(local_order=_empty(n), dp=_empty(n), perm_index=_empty(n), perm_pe=_empty(n),
                   merged_lcp=_empty(n) if merged_lcp else None, local_lcp=_empty(n) if local_lcp else None,
                   intervals=np.zeros(p * p, dtype=np.uint64), recv_counts=np.zeros(p, dtype=np.uint64))
    res = PdResult(_ptr(out["local_order"]), _ptr(out["local_lcp"]), _ptr(out["dp"]), _ptr(out["intervals"]),
                   _ptr(out["perm_index"]), _ptr(out["perm_pe"]), _ptr(out["merged_lcp"]), _ptr(out["recv_counts"]))
    a = ds.arena()
    o = _opts(sampler, 2, small_sort_max, FLAG_LOCAL_LCP if local_lcp else 0)
    check(lib().dsss_pd_sort(ctx.h, ctypes.byref(a), p, _ptr(pb), ctypes.byref(o), ctypes.byref(res),
                             _stream_ptr(stream)))
    out["part_begin"] = pb
    return out


def ms_sort(ctx: Context, ds: DeviceStrings, p: int, part_begin=None, small_sort_max: int = 0, stream=None):
    """DistributedMergeSort::sort on the device: every receiving PE's strings,
    whole and sorted, with LCPs.  Returns torch tensors (device: local_order,
    chars, offsets, lengths, lcp, source) plus host numpy intervals /
    recv_counts and the average LCP."""
    import torch
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    cap = int(ds.lengths[:n].to(torch.int64).sum().item()) + n if n else 0
    # every output byte (strings and their NULs, back to back) is written by the call
    out = dict(local_order=_empty(n), chars=torch.empty(max(cap, 1) + PAD, dtype=torch.uint8, device="cuda"),
               offsets=torch.empty(max(n, 1), dtype=torch.int64, device="cuda"), lengths=_empty(n), lcp=_empty(n),
               source=_empty(n), intervals=np.zeros(p * p, dtype=np.uint64), recv_counts=np.zeros(p, dtype=np.uint64))
    res = MsResult(_ptr(out["local_order"]), _ptr(out["intervals"]), _ptr(out["chars"]), cap, _ptr(out["offsets"]),
                   _ptr(out["lengths"]), _ptr(out["lcp"]), _ptr(out["source"]), _ptr(out["recv_counts"]), 0)
    a = ds.arena()
    o = _opts(0, 2, small_sort_max, 0)
    check(lib().dsss_ms_sort(ctx.h, ctypes.byref(a), p, _ptr(pb), ctypes.byref(o), ctypes.byref(res),
                             _stream_ptr(stream)))
    out["part_begin"] = pb
    out["avg_lcp"] = int(res.avg_lcp)
    out["char_bytes"] = cap
    return out


HQ_SEED = 3469931  # the hQuicksort executable's seed base: PE r seeds its generator with 3469931 + r


def hq_sort(ctx: Context, ds: DeviceStrings, p: int, part_begin=None, seed: int = HQ_SEED, stream=None):
    """RQuick::sort as hQuicksort runs it, on the device: every PE's strings,
    whole and sorted, back to back in rank order.  Returns torch tensors
    (device: chars, offsets, lengths, source) plus host numpy counts (strings
    per PE) and the number of hypercube levels."""
    import torch
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    cap = int(ds.lengths[:n].to(torch.int64).sum().item()) + n if n else 0
    # every output byte (strings and their NULs, back to back) is written by the call
    out = dict(chars=torch.empty(max(cap, 1) + PAD, dtype=torch.uint8, device="cuda"),
               offsets=torch.empty(max(n, 1), dtype=torch.int64, device="cuda"), lengths=_empty(n),
               source=_empty(n), counts=np.zeros(p, dtype=np.uint64))
    res = HqResult(_ptr(out["counts"]), _ptr(out["chars"]), cap, _ptr(out["offsets"]), _ptr(out["lengths"]),
                   _ptr(out["source"]), 0)
    a = ds.arena()
    check(lib().dsss_hq_sort(ctx.h, ctypes.byref(a), p, _ptr(pb), seed, ctypes.byref(res), _stream_ptr(stream)))
    out["part_begin"] = pb
    out["levels"] = int(res.levels)
    out["char_bytes"] = cap
    return out


def distribute_lines(ctx: Context, data, p: int, max_size: int = 0, cap_n: int = None, stream=None):
    """distribute_strings on one GPU: the file bytes `data` (bytes or uint8
    array, pinned for the fastest copy) cut into p PEs' lines ('\\n' -> NUL).
    cap_n: an upper bound on the lines (counted here when not given).
    Returns (DeviceStrings, part_begin)."""
    import torch
    arr = np.frombuffer(data, np.uint8) if isinstance(data, (bytes, bytearray)) else np.ascontiguousarray(data, np.uint8)
    size = int(arr.size)
    S = min(size, max_size) if max_size else size
    if cap_n is None:
        b = arr[:S].tobytes()
        cap_n = b.count(b"\n") + b.count(b"\0") + 1
    cap = S + 1 + PAD
    chars = torch.empty(cap, dtype=torch.uint8, device="cuda")  # the call copies the text and zeroes the rest
    offs = torch.empty(cap_n, dtype=torch.int64, device="cuda")
    lens = torch.empty(cap_n, dtype=torch.int32, device="cuda")
    n, cb = ctypes.c_uint64(0), ctypes.c_uint64(0)
    pb = np.zeros(p + 1, np.uint64)
    check(lib().dsss_distribute_lines(ctx.h, _ptr(arr), size, max_size, p, _ptr(chars), cap, _ptr(offs), _ptr(lens),
                                      cap_n, ctypes.byref(n), ctypes.byref(cb), _ptr(pb), _stream_ptr(stream)))
    ds = DeviceStrings.__new__(DeviceStrings)
    ds.chars, ds.offsets, ds.lengths = chars, offs[:max(n.value, 1)], lens[:max(n.value, 1)]
    ds.char_bytes, ds.n = int(cb.value), int(n.value)
    return ds, pb


def varint_encode(ctx: Context, values, range_counts=None, stream=None):
    """LCPs (device uint32/int32 tensor) to their varint bytes (device uint8
    tensor); with range_counts (values per destination) also the bytes per
    range (host uint64), as writeRanges reports them."""
    import torch
    n = int(values.numel())
    rc = np.zeros(0, np.uint64) if range_counts is None else np.asarray(range_counts, np.uint64)
    rb = np.concatenate([[0], np.cumsum(rc)]).astype(np.uint64)
    nr = int(rc.size)
    tot = ctypes.c_uint64(0)
    per = np.zeros(max(nr, 1), np.uint64)
    check(lib().dsss_varint_encode(ctx.h, _ptr(values), n, _ptr(rb), nr, None, 0, ctypes.byref(tot), _ptr(per),
                                   _stream_ptr(stream)))
    out = torch.zeros(max(tot.value, 1), dtype=torch.uint8, device="cuda")
    check(lib().dsss_varint_encode(ctx.h, _ptr(values), n, _ptr(rb), nr, _ptr(out), out.numel(), ctypes.byref(tot),
                                   _ptr(per), _stream_ptr(stream)))
    return out[:tot.value], per[:nr]


def varint_decode(ctx: Context, data, n: int, stream=None):
    """n varint-coded values (device uint8 tensor) to a device int32 tensor."""
    out = _empty(n)
    check(lib().dsss_varint_decode(ctx.h, _ptr(data) if data.numel() else None, int(data.numel()), _ptr(out), n,
                                   _stream_ptr(stream)))
    return out[:n]


def golomb_param(max_value: int, count: int) -> int:
    """getB of the reference's Golomb coder (dsss_golomb_param)."""
    return int(lib().dsss_golomb_param(max_value, count))


def golomb_param_hashes(count: int, p: int) -> int:
    """b of the hash exchange for count hashes sent to one of p PEs."""
    return int(lib().dsss_golomb_param_hashes(count, p))


def golomb_encode(ctx: Context, values, range_counts, b, stream=None):
    """Golomb/delta blocks (dsss_golomb_encode) of ascending device uint64
    values (a torch int64 tensor viewed as unsigned) in ranges of
    range_counts values with parameters b: (device words, words per range)."""
    import torch
    rc = np.ascontiguousarray(range_counts, dtype=np.uint64)
    bb = np.ascontiguousarray(b, dtype=np.uint64)
    nw = ctypes.c_uint64(0)
    rw = np.zeros(max(len(rc), 1), np.uint64)
    vp = _ptr(values) if values.numel() else None
    check(lib().dsss_golomb_encode(ctx.h, vp, _ptr(rc), len(rc), _ptr(bb), None, 0, ctypes.byref(nw), _ptr(rw),
                                   _stream_ptr(stream)))
    out = torch.empty(max(nw.value, 1), dtype=torch.int64, device=values.device)
    check(lib().dsss_golomb_encode(ctx.h, vp, _ptr(rc), len(rc), _ptr(bb), _ptr(out), nw.value, ctypes.byref(nw),
                                   _ptr(rw), _stream_ptr(stream)))
    return out[:nw.value], rw[:len(rc)]


def golomb_decode(ctx: Context, words, max_blocks: int = 1 << 16, stream=None):
    """Values (device int64 tensor) and values per block of back-to-back
    Golomb/delta blocks (dsss_golomb_decode)."""
    import torch
    n = ctypes.c_uint64(0)
    nb = ctypes.c_uint32(0)
    bc = np.zeros(max(max_blocks, 1), np.uint64)
    wp = _ptr(words) if words.numel() else None
    check(lib().dsss_golomb_decode(ctx.h, wp, int(words.numel()), None, 0, ctypes.byref(n), _ptr(bc), max_blocks,
                                   ctypes.byref(nb), _stream_ptr(stream)))
    out = torch.empty(max(n.value, 1), dtype=torch.int64, device=words.device)
    check(lib().dsss_golomb_decode(ctx.h, wp, int(words.numel()), _ptr(out), n.value, ctypes.byref(n), _ptr(bc),
                                   max_blocks, ctypes.byref(nb), _stream_ptr(stream)))
    return out[:n.value], bc[:nb.value]


def pd_sort_host(ctx: Context, hs: HostStrings, p: int, part_begin=None, sampler: int = 0, merged_lcp: bool = True,
                 out=None, pinned: bool = False, stream=None):
    """The same path with host buffers (copies in and out inside the call)."""
    n = hs.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    if out is None:
        mk = (lambda: _alloc_host(max(n, 1) * 4, np.uint32, pinned)[:max(n, 1)])
        out = dict(local_order=mk(), dp=mk(), perm_index=mk(), perm_pe=mk(), merged_lcp=mk() if merged_lcp else None,
                   local_lcp=None, intervals=np.zeros(p * p, dtype=np.uint64), recv_counts=np.zeros(p, dtype=np.uint64))
    res = PdResult(_ptr(out["local_order"]), None, _ptr(out["dp"]), _ptr(out["intervals"]), _ptr(out["perm_index"]),
                   _ptr(out["perm_pe"]), _ptr(out["merged_lcp"]), _ptr(out["recv_counts"]))
    a = hs.arena()
    o = _opts(sampler)
    check(lib().dsss_pd_sort_host(ctx.h, ctypes.byref(a), p, _ptr(pb), ctypes.byref(o), ctypes.byref(res),
                                  _stream_ptr(stream)))
    out["part_begin"] = pb
    return out


def pd_sort_batched(ctx: Context, ds: DeviceStrings, nsets: int, p: int, part_begin, sampler: int = 0,
                    merged_lcp: bool = True, local_lcp: bool = False, small_sort_max: int = 0, stream=None, out=None):
    """dsss_pd_sort_batched: nsets independent sets of p PEs in one arena
    (part_begin: nsets*p + 1 PE bounds, e.g. batched_parts)."""
    n = ds.n
    pb = np.asarray(part_begin, dtype=np.uint64)
    npe = nsets * p
    if out is None:
        out = dict(local_order=_empty(n), dp=_empty(n), perm_index=_empty(n), perm_pe=_empty(n),
                   merged_lcp=_empty(n) if merged_lcp else None, local_lcp=_empty(n) if local_lcp else None,
                   intervals=np.zeros(npe * p, dtype=np.uint64), recv_counts=np.zeros(npe, dtype=np.uint64))
    res = PdResult(_ptr(out["local_order"]), _ptr(out["local_lcp"]), _ptr(out["dp"]), _ptr(out["intervals"]),
                   _ptr(out["perm_index"]), _ptr(out["perm_pe"]), _ptr(out["merged_lcp"]), _ptr(out["recv_counts"]))
    o = _opts(sampler, 2, small_sort_max, FLAG_LOCAL_LCP if local_lcp else 0)
    check(lib().dsss_pd_sort_batched(ctx.h, ctypes.byref(ds.arena()), nsets, p, _ptr(pb), ctypes.byref(o),
                                     ctypes.byref(res), _stream_ptr(stream)))
    out["part_begin"] = pb
    return out


def pd_sort_batched_host(ctx: Context, hs: HostStrings, nsets: int, p: int, part_begin, sampler: int = 0,
                         merged_lcp: bool = True, out=None, pinned: bool = False, stream=None):
    """dsss_pd_sort_batched_host: the batched path with host buffers."""
    n = hs.n
    pb = np.asarray(part_begin, dtype=np.uint64)
    npe = nsets * p
    if out is None:
        mk = (lambda: _alloc_host(max(n, 1) * 4, np.uint32, pinned)[:max(n, 1)])
        out = dict(local_order=mk(), dp=mk(), perm_index=mk(), perm_pe=mk(), merged_lcp=mk() if merged_lcp else None,
                   local_lcp=None, intervals=np.zeros(npe * p, dtype=np.uint64),
                   recv_counts=np.zeros(npe, dtype=np.uint64))
    res = PdResult(_ptr(out["local_order"]), None, _ptr(out["dp"]), _ptr(out["intervals"]), _ptr(out["perm_index"]),
                   _ptr(out["perm_pe"]), _ptr(out["merged_lcp"]), _ptr(out["recv_counts"]))
    check(lib().dsss_pd_sort_batched_host(ctx.h, ctypes.byref(hs.arena()), nsets, p, _ptr(pb),
                                          ctypes.byref(_opts(sampler)), ctypes.byref(res), _stream_ptr(stream)))
    out["part_begin"] = pb
    return out


TUNE_KNOBS = ("dp_filter_min", "dp_filter_bits", "sort_small_max", "sort_pivot", "dp_table", "sort_graph_max_n", "merge_by_sort",
              "merge_extend_lanes", "dp_split", "copy_word", "dp_digest", "dp_check", "sort_split_min", "sort_bits",
              "sort_seg_bits")


def tune_set(name: str, value: int):
    """Sets a process-wide tuning knob (-1 restores its default)."""
    check(lib().dsss_tune_set(name.encode(), int(value)))


def tune_get(name: str) -> int:
    v = ctypes.c_int64(0)
    check(lib().dsss_tune_get(name.encode(), ctypes.byref(v)))
    return int(v.value)


class tuned:
    """Context manager: knobs set for the block, defaults restored after."""

    def __init__(self, **knobs):
        self.knobs = knobs

    def __enter__(self):
        self.old = {k: tune_get(k) for k in self.knobs}
        for k, v in self.knobs.items():
            tune_set(k, v)
        return self

    def __exit__(self, *exc):
        for k, v in self.old.items():
            tune_set(k, v)


def autotune(ctx: Context, ds, p: int, part_begin=None, nsets: int = 1, sampler: int = 0, trials: int = 2,
             stream=None) -> dict:
    """dsss_autotune on this input: times the knob grid and leaves the fastest
    setting in force; returns it with its time and the default's."""
    pb = equal_parts(ds.n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    t = Tuning()
    check(lib().dsss_autotune(ctx.h, ctypes.byref(ds.arena()), nsets, p, _ptr(pb), ctypes.byref(_opts(sampler)),
                              trials, ctypes.byref(t), _stream_ptr(stream)))
    return {k: getattr(t, k) for k, _ in Tuning._fields_}


def clock_now() -> float:
    """The server's clock (steady, seconds)."""
    return float(lib().dsss_clock_now())


class Server:
    """dsss_server: continuous batching of sort requests onto one GPU."""

    def __init__(self, device: int = 0, p: int = 4, workers: int = 2, max_sets: int = 0, max_batch_strings: int = 0,
                 hbm_budget: int = 0, sampler: int = 0, small_sort_max: int = 0, timestamps: bool = False,
                 reserve_bytes: int = 0):
        cfg = ServerConfig(device, workers, p, max_sets, max_batch_strings, hbm_budget, _opts(sampler, 2, small_sort_max),
                           1 if timestamps else 0, reserve_bytes)
        h = ctypes.c_void_p()
        check(lib().dsss_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.p = p
        self._live = {}

    def submit(self, hs: HostStrings, part_begin=None, merged_lcp: bool = True, out=None):
        """Queues one request; returns (ticket, out) with out's host arrays
        filled once wait(ticket) returns."""
        n, p = hs.n, self.p
        if out is None:
            mk = (lambda: np.empty(max(n, 1), np.uint32))
            out = dict(local_order=mk(), dp=mk(), perm_index=mk(), perm_pe=mk(),
                       merged_lcp=mk() if merged_lcp else None, intervals=np.zeros(p * p, np.uint64),
                       recv_counts=np.zeros(p, np.uint64))
        pb = None if part_begin is None else np.ascontiguousarray(part_begin, dtype=np.uint64)
        res = PdResult(_ptr(out["local_order"]), None, _ptr(out["dp"]), _ptr(out["intervals"]),
                       _ptr(out["perm_index"]), _ptr(out["perm_pe"]), _ptr(out["merged_lcp"]),
                       _ptr(out["recv_counts"]))
        a = hs.arena()
        t = ctypes.c_uint64(0)
        check(lib().dsss_server_submit(self.h, ctypes.byref(a), _ptr(pb), ctypes.byref(res), ctypes.byref(t)))
        out["part_begin"] = pb if pb is not None else equal_parts(n, p)
        self._live[t.value] = (hs, out, pb)
        return t.value, out

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        st = RequestStats()
        rc = lib().dsss_server_wait(self.h, ticket, timeout_ms, ctypes.byref(st))
        if rc == -110:
            check(rc)
        self._live.pop(ticket, None)
        check(rc)
        return dict(batch_sets=st.batch_sets, batch_id=st.batch_id, batch_strings=st.batch_strings,
                    t_submit=st.t_submit, t_admit=st.t_admit, t_done=st.t_done, t_copied=st.t_copied,
                    t_sorted=st.t_sorted,
                    latency=st.t_done - st.t_submit)

    def info(self) -> dict:
        i = ServerInfo()
        check(lib().dsss_server_info(self.h, ctypes.byref(i)))
        return {k: int(getattr(i, k)) for k, _ in ServerInfo._fields_}

    def footprint(self, n: int, char_bytes: int) -> int:
        return int(lib().dsss_server_footprint(self.h, n, char_bytes))

    def close(self):
        if self.h:
            check(lib().dsss_server_destroy(self.h))
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def local_sort_lcp(ctx: Context, ds: DeviceStrings, p: int = 1, part_begin=None, small_sort_max: int = 0,
                   stream=None):
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    order, lcp = _empty(n), _empty(n)
    o = _opts(small_sort_max=small_sort_max)
    check(lib().dsss_local_sort_lcp(ctx.h, ctypes.byref(ds.arena()), p, _ptr(pb), ctypes.byref(o), _ptr(order),
                                    _ptr(lcp), _stream_ptr(stream)))
    return order[:n], lcp[:n]


def dp_prefixes(ctx: Context, ds: DeviceStrings, order, lcp, p: int = 1, part_begin=None, max_rounds: int = 64,
                stream=None):
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    dp = _empty(n)
    counts = np.zeros(max_rounds, dtype=np.uint64)
    rounds = ctypes.c_uint32(0)
    check(lib().dsss_dp_prefixes(ctx.h, ctypes.byref(ds.arena()), p, _ptr(pb), _ptr(order), _ptr(lcp), _ptr(dp),
                                 _ptr(counts), max_rounds, ctypes.byref(rounds), _stream_ptr(stream)))
    return dp[:n], counts[:rounds.value]


def dp_round(ctx: Context, ds: DeviceStrings, order, lcp, candidates, depth: int, results, stream=None):
    """One BloomFilter::filter round (dsss_dp_round): returns (next positions, count)."""
    n = ds.n
    nxt = _empty(n)
    m = 0 if candidates is None else int(candidates.shape[0])
    mn = np.zeros(1, dtype=np.uint64)
    check(lib().dsss_dp_round(ctx.h, ctypes.byref(ds.arena()), _ptr(order), _ptr(lcp), _ptr(candidates), m, depth,
                              _ptr(results), _ptr(nxt), _ptr(mn), _stream_ptr(stream)))
    return nxt[:int(mn[0])], int(mn[0])


def bucket_scatter(ctx: Context, ds: DeviceStrings, p: int, local_order, lcp, dp, intervals, part_begin=None,
                   stream=None):
    """dsss_bucket_scatter: every PE's receive container, back to back."""
    import torch
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    iv = np.ascontiguousarray(np.asarray(intervals, dtype=np.uint64).ravel())
    total = np.zeros(1, np.uint64)
    cbeg = np.zeros(p + 1, np.uint64)
    counts = np.zeros(p * p, np.uint64)
    offs = np.zeros(p * p, np.uint64)
    cstart, rl, ri, rp = _empty(n), _empty(n), _empty(n), _empty(n)
    args = [ctx.h, ctypes.byref(ds.arena()), p, _ptr(pb), _ptr(local_order), _ptr(lcp), _ptr(dp), _ptr(iv)]
    check(lib().dsss_bucket_scatter(*args, None, 0, _ptr(total), _ptr(cbeg), None, _ptr(rl), _ptr(ri), _ptr(rp),
                                    _ptr(counts), _ptr(offs), _stream_ptr(stream)))
    chars = torch.zeros(int(total[0]) + PAD, dtype=torch.uint8, device=ds.chars.device)
    check(lib().dsss_bucket_scatter(*args, _ptr(chars), int(total[0]) + PAD, _ptr(total), _ptr(cbeg), _ptr(cstart),
                                    _ptr(rl), _ptr(ri), _ptr(rp), _ptr(counts), _ptr(offs), _stream_ptr(stream)))
    return dict(chars=chars, char_total=int(total[0]), char_begin=cbeg, char_start=cstart[:n], lcp=rl[:n],
                index=ri[:n], pe=rp[:n], counts=counts.reshape(p, p), offsets=offs.reshape(p, p))


def lcp_merge(ctx: Context, chars, char_bytes: int, lcp, counts, offsets=None, char_start=None, stream=None):
    """dsss_lcp_merge over nrecv x p source runs (counts/offsets shaped (nrecv, p))."""
    counts = np.ascontiguousarray(np.asarray(counts, dtype=np.uint64))
    nrecv, p = counts.shape
    offs = None if offsets is None else np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
    n = int(lcp.shape[0])
    out = dict(order=_empty(n), merged_lcp=_empty(n), old_lcp=_empty(n), perm_index=_empty(n), perm_pe=_empty(n))
    check(lib().dsss_lcp_merge(ctx.h, _ptr(chars), char_bytes, _ptr(char_start), _ptr(lcp), n, nrecv, p, _ptr(counts),
                               _ptr(offs), _ptr(out["order"]), _ptr(out["merged_lcp"]), _ptr(out["old_lcp"]),
                               _ptr(out["perm_index"]), _ptr(out["perm_pe"]), _stream_ptr(stream)))
    return {k: v[:n] for k, v in out.items()}


def lcp_merge_strings(ctx: Context, chars, char_bytes: int, lcp, counts, offsets=None, char_start=None,
                      lcp_sum: int = None, stream=None):
    """dsss_lcp_merge_strings: the merge of receive containers of whole strings
    and every merged string whole, back to back in merged order.  lcp_sum (the
    sum of lcp; read from the device when not given) sizes the output.
    Returns device tensors chars, offsets, lengths, merged_lcp, order."""
    import torch
    counts = np.ascontiguousarray(np.asarray(counts, dtype=np.uint64))
    nrecv, p = counts.shape
    offs = None if offsets is None else np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
    n = int(lcp.shape[0])
    if lcp_sum is None:
        lcp_sum = int(lcp[:n].to(torch.int64).sum().item()) if n else 0
    cap = char_bytes + lcp_sum
    out = dict(order=_empty(n), merged_lcp=_empty(n), lengths=_empty(n),
               offsets=torch.empty(max(n, 1), dtype=torch.int64, device="cuda"),
               chars=torch.empty(max(cap, 1) + PAD, dtype=torch.uint8, device="cuda"))
    nb = ctypes.c_uint64(0)
    check(lib().dsss_lcp_merge_strings(ctx.h, _ptr(chars), char_bytes, _ptr(char_start), _ptr(lcp), n, nrecv, p,
                                       _ptr(counts), _ptr(offs), _ptr(out["order"]), _ptr(out["merged_lcp"]),
                                       _ptr(out["chars"]), cap, _ptr(out["offsets"]), _ptr(out["lengths"]),
                                       ctypes.byref(nb), _stream_ptr(stream)))
    res = {k: out[k][:n] for k in ("order", "merged_lcp", "lengths", "offsets")}
    res["chars"] = out["chars"]
    res["char_bytes"] = int(nb.value)
    return res


def prefix_hash(ds: DeviceStrings, ids, depth: int, stream=None):
    import torch
    m = int(ids.shape[0])
    out = torch.empty(max(m, 1), dtype=torch.int64, device=ids.device)
    check(lib().dsss_prefix_hash(ctypes.byref(ds.arena()), _ptr(ids), m, depth, _ptr(out), _stream_ptr(stream)))
    return out[:m]


def partition(ctx: Context, ds: DeviceStrings, order, dp, p: int, part_begin=None, sampler: int = 0, stream=None):
    n = ds.n
    pb = equal_parts(n, p) if part_begin is None else np.asarray(part_begin, dtype=np.uint64)
    iv = np.zeros(p * p, dtype=np.uint64)
    o = _opts(sampler)
    check(lib().dsss_partition(ctx.h, ctypes.byref(ds.arena()), p, _ptr(pb), _ptr(order), _ptr(dp), ctypes.byref(o),
                               _ptr(iv), _stream_ptr(stream)))
    return iv.reshape(p, p)


def adjacent_lcp_noalloc(ds: DeviceStrings, order, lcp, stream=None):
    """dsss_adjacent_lcp_noalloc: writes into the caller's lcp tensor and
    allocates nothing (see include/dsss.h)."""
    m = int(order.shape[0])
    # the entry point trusts its pointers: a short or host-side output would
    # be written out of bounds on the device
    if not (getattr(lcp, "is_cuda", False) and getattr(order, "is_cuda", False)):
        raise ValueError("order and lcp must be CUDA tensors")
    if lcp.device != order.device or ds.chars.device != order.device:
        raise ValueError("order, lcp and the strings must be on one device")
    import torch
    if lcp.dtype != torch.int32 or order.dtype != torch.int32:
        raise ValueError("order and lcp must be int32 tensors")
    if lcp.numel() < m or not lcp.is_contiguous() or not order.is_contiguous():
        raise ValueError("lcp needs at least len(order) contiguous entries")
    check(lib().dsss_adjacent_lcp_noalloc(ctypes.byref(ds.arena()), _ptr(order), m, _ptr(lcp), _stream_ptr(stream)))
    return lcp


def adjacent_lcp(ctx: Context, ds: DeviceStrings, order, stream=None):
    m = int(order.shape[0])
    out = _empty(m)
    check(lib().dsss_adjacent_lcp(ctx.h, ctypes.byref(ds.arena()), _ptr(order), m, _ptr(out), _stream_ptr(stream)))
    return out[:m]
