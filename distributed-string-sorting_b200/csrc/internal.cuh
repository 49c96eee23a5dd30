// Shared internals of libdsss: context, error reporting, scratch carving and
// the device helpers every kernel uses (big-endian 8-byte key loads, XXH64).
#pragma once
#include <atomic>

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/dsss.h"

namespace dsss {

// ---------------------------------------------------------------- errors ----
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define DSSS_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::dsss::fail(DSSS_EDEVICE, "%s:%d %s: %s", __FILE__, __LINE__, #call,    \
                                cudaGetErrorString(e_));                                  \
    } while (0)

#define DSSS_TRY(expr)             \
    do {                           \
        int r_ = (expr);           \
        if (r_ != DSSS_OK) return r_; \
    } while (0)

// --------------------------------------------------------------- context ----
// Per-kernel timing: when a context has timing on, every launch made through
// DSSS_LAUNCH inside its calls is bracketed by CUDA events on the launching
// stream; durations are folded into per-name totals when the call finishes.
struct KernelTimes {
    bool on = false;
    struct Pending { const char* name; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    std::vector<std::string> names;
    std::vector<double> total_ms;
    std::vector<uint64_t> launches;
    cudaEvent_t get();
    void fold();  // after the stream has been synchronised
};

struct Ctx {
    int device = 0;
    uint64_t budget = 0;     // 0 = unlimited
    void* ws = nullptr;      // device scratch, grown on demand
    uint64_t ws_cap = 0;
    bool fixed_ws = false;   // ws is a block of someone else's buffer: never reallocated
    void* pin = nullptr;     // pinned host staging for small read-backs
    uint64_t pin_cap = 0;
    KernelTimes* times = nullptr;
};

// The context whose call is running on this thread (for launch timing).
extern thread_local KernelTimes* g_times;
struct ActiveCtx {
    KernelTimes* prev;
    explicit ActiveCtx(Ctx* c) : prev(g_times) { g_times = (c && c->times && c->times->on) ? c->times : nullptr; }
    ~ActiveCtx() { g_times = prev; }
};

// Brackets a stage (several launches and host read-backs) the same way.
struct StageTimer {
    KernelTimes* kt;
    const char* name;
    cudaEvent_t a = nullptr;
    cudaStream_t st;
    StageTimer(const char* nm, cudaStream_t s) : kt(g_times), name(nm), st(s) {
        if (kt) { a = kt->get(); cudaEventRecord(a, st); }
    }
    void end() {
        if (kt) {
            cudaEvent_t b = kt->get();
            cudaEventRecord(b, st);
            kt->pending.push_back({name, a, b});
            kt = nullptr;
        }
    }
    ~StageTimer() { end(); }
};

#define DSSS_LAUNCH(name, st, ...)                                          \
    do {                                                                    \
        ::dsss::KernelTimes* kt_ = ::dsss::g_times;                         \
        cudaEvent_t a_ = nullptr, b_ = nullptr;                             \
        if (kt_) { a_ = kt_->get(); b_ = kt_->get(); cudaEventRecord(a_, st); } \
        __VA_ARGS__;                                                        \
        if (kt_) { cudaEventRecord(b_, st); kt_->pending.push_back({name, a_, b_}); } \
    } while (0)

// Bump allocator over the context scratch.  Run a layout twice: first with
// sizing = true to learn the total, then for real after ensure_ws().
struct Carve {
    char* base;
    uint64_t used = 0;
    bool sizing;
    explicit Carve(void* b) : base((char*)b), sizing(b == nullptr) {}
    template <typename T>
    T* take(uint64_t count) {
        used = (used + 255) & ~255ull;
        T* p = sizing ? nullptr : (T*)(base + used);
        used += count * sizeof(T);
        return p;
    }
};

// Raises a kernel's dynamic shared-memory limit once per device.  Safe from
// several host threads: concurrent first calls both set it, which is harmless.
template <typename K>
inline int set_smem_once(std::atomic<uint64_t>& done, K* kernel, int bytes) {
    int dev = 0;
    DSSS_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return DSSS_OK;
    DSSS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done.fetch_or(bit, std::memory_order_release);
    return DSSS_OK;
}

// Process-wide tuning knobs (dsss_tune_set / dsss_tune_get), read at call time.
enum TuneKnob : int {
    TUNE_DP_FILTER_MIN = 0,  // hashed strings per round from which the fingerprint filter is used
    TUNE_DP_FILTER_BITS,     // filter bits per hashed string (rounded up to a power of two in total)
    TUNE_SORT_SMALL_MAX,     // small-segment cutoff when the options give 0
    TUNE_SORT_PIVOT,         // pivot passes on (1) or off (0)
    TUNE_DP_TABLE,           // DP hash-table slots per hashed string (rounded up to a power of two)
    TUNE_SORT_GRAPH,         // largest n sorted by the device-driven graph (0: never)
    TUNE_MERGE_SORT,         // receive containers merged by sorting their union (1), by merge rounds (0) or
                             // by co-ranked tiles of all runs at once (2)
    TUNE_MERGE_LANES,        // threads per chunk of strings in the prefix decompression (0: from the length)
    TUNE_DP_SPLIT,           // hash round split into hashing and table inserts (1) or one kernel (0)
    TUNE_COPY_WORD,          // bytes per store when whole strings are copied out (16, or 8)
    TUNE_DP_DIGEST,          // hash rounds in which at least 1/k of the positions hash run in arena order
                             // (k_dp_arena_insert); 0 turns the arena-order form off
    TUNE_DP_CHECK,           // 1: the arena-order rounds recompute every stored prefix hash from the string and
                             // fail on a mismatch (a self-check)
    TUNE_SORT_SPLIT_MIN,     // smallest large segment that may split by sampled splitters instead of a key
                             // byte (0: never, the default; values below 4096 count as 4096)
    TUNE_SORT_BITS,          // 1: passes over plain keys split on the keys' eight most significant differing
                             // bits (several key bytes over small alphabets); 2: only where the first
                             // differing byte varies in at most four bits; 3: the same in the first pass
                             // only; 0: on one key byte (default)
    TUNE_SORT_SEG_BITS,      // the same for the shared-memory passes of the segment sorter (default 0)
    TUNE_COUNT
};
int64_t tune(TuneKnob k);

int ensure_ws(Ctx* c, uint64_t bytes);
int ensure_pin(Ctx* c, uint64_t bytes);

// ------------------------------------------------------------ arena view ----
struct ArenaDev {
    const uint8_t* chars;
    const uint64_t* off;
    const uint32_t* len;
    uint64_t n;
    // Optional interleaved (offset, length) per string: one 16-byte load (one
    // memory sector) per random lookup instead of two.
    const ulonglong2* h = nullptr;
};

// Offset and length of string s.
__device__ __forceinline__ void str_of(const ArenaDev& a, uint32_t s, uint64_t& off, uint32_t& len) {
    if (a.h) {
        const ulonglong2 v = __ldg(&a.h[s]);
        off = v.x;
        len = (uint32_t)v.y;
    } else {
        off = a.off[s];
        len = a.len[s];
    }
}

// Builds the interleaved handle array for strings [0, n).
void make_handles(const ArenaDev& a, ulonglong2* h, cudaStream_t st);

int check_arena(const dsss_arena* a);

// --------------------------------------------------------- device helpers ----
__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | (uint64_t)__byte_perm(hi, 0, 0x0123);
}

// 8 bytes at an arbitrary address as a little-endian word, from two aligned
// 8-byte loads.  Reads up to 15 bytes past p; the arena contract pads 32.
__device__ __forceinline__ uint64_t load_le8(const uint8_t* p) {
    uintptr_t a = (uintptr_t)p;
    const unsigned long long* q = (const unsigned long long*)(a & ~(uintptr_t)7);
    unsigned sh = (unsigned)(a & 7) * 8;
    uint64_t lo = __ldg(q);
    if (sh == 0) return lo;
    uint64_t hi = __ldg(q + 1);
    return (lo >> sh) | (hi << (64 - sh));
}

// Copies len bytes from src to dst with L lanes (lane = 0..L-1 of the
// calling group): dst's aligned 8-byte words are stored whole, each from an
// unaligned 8-byte load of src (reads at most 15 bytes past src + len; the
// arena contract pads 32), the at most 7 bytes before and after them singly.
template <uint32_t L>
__device__ __forceinline__ void copy_words(uint8_t* dst, const uint8_t* src, uint32_t len, uint32_t lane) {
    const uintptr_t d0 = (uintptr_t)dst, e = d0 + len;
    const uintptr_t a0 = (d0 + 7) & ~(uintptr_t)7, a1 = e & ~(uintptr_t)7;
    if (a0 >= a1) {
        for (uint32_t k = lane; k < len; k += L) dst[k] = src[k];
        return;
    }
    const uint32_t head = (uint32_t)(a0 - d0), tail = (uint32_t)(a1 - d0);
    for (uint32_t k = lane; k < head; k += L) dst[k] = src[k];
    for (uint32_t k = tail + lane; k < len; k += L) dst[k] = src[k];
    const uint32_t nw = (uint32_t)((a1 - a0) >> 3);
    unsigned long long* w = reinterpret_cast<unsigned long long*>(a0);
#pragma unroll 4
    for (uint32_t k = lane; k < nw; k += L) w[k] = load_le8(src + head + 8 * k);
}

// copy_words with dst's aligned 16-byte words stored whole, each from three
// aligned 8-byte loads of src (reads at most 8 bytes past src + len), the at
// most 15 bytes before and after them singly.
template <uint32_t L>
__device__ __forceinline__ void copy_words16(uint8_t* dst, const uint8_t* src, uint32_t len, uint32_t lane) {
    const uintptr_t d0 = (uintptr_t)dst, e = d0 + len;
    const uintptr_t a0 = (d0 + 15) & ~(uintptr_t)15, a1 = e & ~(uintptr_t)15;
    if (a0 >= a1) {
        for (uint32_t k = lane; k < len; k += L) dst[k] = src[k];
        return;
    }
    const uint32_t head = (uint32_t)(a0 - d0), tail = (uint32_t)(a1 - d0);
    for (uint32_t k = lane; k < head; k += L) dst[k] = src[k];
    for (uint32_t k = tail + lane; k < len; k += L) dst[k] = src[k];
    const uint32_t nw = (uint32_t)((a1 - a0) >> 4);
    uint4* w = reinterpret_cast<uint4*>(a0);
    const uintptr_t sa = (uintptr_t)(src + head);
    const unsigned long long* q = reinterpret_cast<const unsigned long long*>(sa & ~(uintptr_t)7);
    const unsigned sh = (unsigned)(sa & 7) * 8;
#pragma unroll 2
    for (uint32_t k = lane; k < nw; k += L) {
        const uint64_t x0 = __ldg(q + 2 * k), x1 = __ldg(q + 2 * k + 1);
        uint64_t lo = x0, hi = x1;
        if (sh) {
            const uint64_t x2 = __ldg(q + 2 * k + 2);
            lo = (x0 >> sh) | (x1 << (64 - sh));
            hi = (x1 >> sh) | (x2 << (64 - sh));
        }
        w[k] = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
    }
}

// Bytes [depth, depth+8) of a string as a big-endian key; bytes at or past
// the string's length are 0 (the NUL terminator and beyond), so unsigned key
// order is the reference's byte-wise string order (scmp, stringtools.hpp:128).
__device__ __forceinline__ uint64_t key8(const uint8_t* chars, uint64_t off, uint32_t len,
                                         uint32_t depth) {
    if (depth >= len) return 0;
    uint64_t v = load_le8(chars + off + depth);
    uint32_t rem = len - depth;
    if (rem < 8) v &= (1ull << (rem * 8)) - 1;
    return bswap64(v);
}

__device__ __forceinline__ uint64_t key8_of(const ArenaDev& a, uint32_t s, uint32_t depth) {
    uint64_t off;
    uint32_t len;
    str_of(a, s, off, len);
    return key8(a.chars, off, len, depth);
}

// Index (0..7) of the first zero byte of a big-endian key, or 8 if none.
__device__ __forceinline__ uint32_t zero_byte(uint64_t k) {
    const uint64_t m = 0x7F7F7F7F7F7F7F7Full;
    // Exact per-byte zero test (no borrow between bytes): 0x80 in each zero byte.
    uint64_t z = ~(((k & m) + m) | k | m);
    return z ? (uint32_t)(__clzll(z) >> 3) : 8u;
}

// LCP in bytes of two keys that differ.
__device__ __forceinline__ uint32_t key_lcp(uint64_t a, uint64_t b) {
    return (uint32_t)(__clzll(a ^ b) >> 3);
}

// --------------------------------------------------------------- XXH64 ----
// XXH64, seed 0, of m bytes at p: the published algorithm as the reference's
// streaming port computes it (hash/xxhash.hpp:327-350, 516-660), including the
// port's "total_len > 32" choice of the four-lane merge (xxhash.hpp:608).
namespace xxh {
constexpr uint64_t P1 = 11400714785074694791ULL, P2 = 14029467366897019727ULL,
                   P3 = 1609587929392839161ULL, P4 = 9650029242287828579ULL,
                   P5 = 2870177450012600261ULL;
__device__ __forceinline__ uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
__device__ __forceinline__ uint64_t round(uint64_t acc, uint64_t in) {
    acc += in * P2;
    acc = rotl(acc, 31);
    return acc * P1;
}
__device__ __forceinline__ uint64_t merge(uint64_t acc, uint64_t v) {
    v = round(0, v);
    acc ^= v;
    return acc * P1 + P4;
}
}  // namespace xxh

// Streams little-endian 8-byte words from an unaligned start with one aligned
// 16-byte load per two words.
struct WordStream {
    const uint4* q;
    unsigned sh;
    uint64_t w0, w1, w2;  // w0 current aligned word, w1/w2 buffered
    int buffered;         // words buffered after w0
    __device__ __forceinline__ explicit WordStream(const uint8_t* p) {
        uintptr_t a = (uintptr_t)p;
        sh = (unsigned)(a & 7) * 8;
        uintptr_t wa = a & ~(uintptr_t)7;           // first aligned word
        q = (const uint4*)(wa & ~(uintptr_t)15);
        uint4 v = __ldg(q++);
        uint64_t lo = ((uint64_t)v.y << 32) | v.x, hi = ((uint64_t)v.w << 32) | v.z;
        if (wa & 8) { w0 = hi; buffered = 0; }
        else { w0 = lo; w1 = hi; buffered = 1; }
    }
    __device__ __forceinline__ uint64_t next_aligned() {
        if (buffered == 0) {
            uint4 v = __ldg(q++);
            w1 = ((uint64_t)v.y << 32) | v.x;
            w2 = ((uint64_t)v.w << 32) | v.z;
            buffered = 2;
        }
        uint64_t r = w1;
        w1 = w2;
        --buffered;
        return r;
    }
    __device__ __forceinline__ uint64_t next() {
        uint64_t lo = w0;
        uint64_t hi = next_aligned();
        w0 = hi;
        return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
    }
};

// XXH64 of m <= XXH_SHORT_MAX bytes at p with all of its 16-byte loads
// issued before the first round, so that they are in flight together (the
// streaming form below waits for each load in turn).  Same value as the
// streaming form.  Reads up to 22 bytes past p + m.
constexpr uint32_t XXH_SHORT_MAX = 88;
__device__ __forceinline__ uint64_t xxh64_short(const uint8_t* p, uint32_t m) {
    using namespace xxh;
    const uintptr_t a = (uintptr_t)p;
    const uint4* q = (const uint4*)(a & ~(uintptr_t)15);
    const uint32_t skip = (uint32_t)(a & 15);
    const uint32_t nq = (skip + m + 8 + 15) / 16;  // chunks up to byte p + m + 7
    uint64_t w[14];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if ((uint32_t)k < nq) v = __ldg(q + k);
        w[2 * k] = ((uint64_t)v.y << 32) | v.x;
        w[2 * k + 1] = ((uint64_t)v.w << 32) | v.z;
    }
    const bool odd = skip >= 8;
    const uint32_t sh = (skip & 7) * 8;
    // input word j = bytes [p + 8j, p + 8j + 8), little-endian
    auto word = [&](int j) -> uint64_t {
        const uint64_t lo = odd ? w[j + 1] : w[j];
        const uint64_t hi = odd ? w[j + 2] : w[j + 1];
        return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
    };
    const uint32_t ns = m >= 64 ? 2u : (m >= 32 ? 1u : 0u);  // 32-byte stripes
    uint64_t v1 = P1 + P2, v2 = P2, v3 = 0, v4 = 0 - P1;
    if (ns >= 1) {
        v1 = round(v1, word(0));
        v2 = round(v2, word(1));
        v3 = round(v3, word(2));
        v4 = round(v4, word(3));
    }
    if (ns >= 2) {
        v1 = round(v1, word(4));
        v2 = round(v2, word(5));
        v3 = round(v3, word(6));
        v4 = round(v4, word(7));
    }
    uint64_t h;
    if (m > 32) {
        h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
        h = merge(h, v1);
        h = merge(h, v2);
        h = merge(h, v3);
        h = merge(h, v4);
    } else {
        h = v3 + P5;
    }
    h += m;
    const uint32_t t0 = 4 * ns, t1 = t0 + (m - 32 * ns) / 8;  // 8-byte tail words [t0, t1)
    uint32_t rem = (m - 32 * ns) & 7;
    uint64_t last = 0;
#pragma unroll
    for (int j = 0; j < 11; ++j) {
        const uint64_t x = word(j);
        if ((uint32_t)j >= t0 && (uint32_t)j < t1) {
            h ^= round(0, x);
            h = rotl(h, 27) * P1 + P4;
        }
        if ((uint32_t)j == t1) last = x;
    }
    if (rem) {
        uint64_t wv = last;  // bytes past m are ignored
        if (rem >= 4) {
            h ^= (uint64_t)(uint32_t)wv * P1;
            h = rotl(h, 23) * P2 + P3;
            wv >>= 32;
            rem -= 4;
        }
        while (rem) {
            h ^= (wv & 0xff) * P5;
            h = rotl(h, 11) * P1;
            wv >>= 8;
            --rem;
        }
    }
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
}

__device__ __forceinline__ uint64_t xxh64_dev(const uint8_t* p, uint32_t m) {
    using namespace xxh;
    if (m <= XXH_SHORT_MAX) return xxh64_short(p, m);
    WordStream ws(p);
    uint64_t v1 = P1 + P2, v2 = P2, v3 = 0, v4 = 0 - P1;
    uint32_t rem = m;
    if (m >= 32) {
        do {
            v1 = round(v1, ws.next());
            v2 = round(v2, ws.next());
            v3 = round(v3, ws.next());
            v4 = round(v4, ws.next());
            rem -= 32;
        } while (rem >= 32);
    }
    uint64_t h;
    if (m > 32) {
        h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
        h = merge(h, v1);
        h = merge(h, v2);
        h = merge(h, v3);
        h = merge(h, v4);
    } else {
        h = v3 + P5;
    }
    h += m;
    while (rem >= 8) {
        h ^= round(0, ws.next());
        h = rotl(h, 27) * P1 + P4;
        rem -= 8;
    }
    if (rem) {
        uint64_t w = ws.next();  // bytes past m are ignored
        if (rem >= 4) {
            h ^= (uint64_t)(uint32_t)w * P1;
            h = rotl(h, 23) * P2 + P3;
            w >>= 32;
            rem -= 4;
        }
        while (rem) {
            h ^= (w & 0xff) * P5;
            h = rotl(h, 11) * P1;
            w >>= 8;
            --rem;
        }
    }
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
}

// XXHasher::hash with bloomFilterSize = UINT64_MAX (bloomfilter.hpp:1094-1102, :1135).
__device__ __forceinline__ uint64_t filter_hash(uint64_t h) { return h == ~0ull ? 0 : h; }

// The first four depths of the distinguishing-prefix schedule (8, 24, 40,
// 72): the string sort's first pass, which reads every string's first bytes
// in arena order anyway, stores each string's filter hashes at these depths
// so that a dense hash round at one of them reads 8 bytes per string instead
// of the prefix.
constexpr int ROOT_DIGESTS = 4;
__host__ __device__ constexpr uint32_t root_digest_depth(int j) { return j == 0 ? 8u : j == 1 ? 24u : j == 2 ? 40u : 72u; }
__host__ __device__ inline int root_digest_index(uint64_t depth) {
    return depth == 8 ? 0 : depth == 24 ? 1 : depth == 40 ? 2 : depth == 72 ? 3 : -1;
}

// filter_hash(XXH64(p, d)) for the depths d = 8, 24, 40, 72 whose bit is set
// in want, from one set of loads (the words of the first 72 bytes); out[j]
// for depths beyond len, or not wanted, is left as is.  The same values as
// xxh64_dev (one stripe feeds the 40-byte hash, two the 72-byte one; both
// merge the lanes since their lengths exceed 32).
__device__ __forceinline__ void root_digests(const uint8_t* p, uint32_t len, unsigned long long* out,
                                             uint64_t stride, uint32_t want) {
    using namespace xxh;
    if (len < 8 || !want) return;
    const uintptr_t a = (uintptr_t)p;
    const uint4* q = (const uint4*)(a & ~(uintptr_t)15);
    const uint32_t skip = (uint32_t)(a & 15);
    const uint32_t m = len < 72 ? len : 72;
    const uint32_t nq = (skip + m + 15) / 16;  // chunks up to byte p + m - 1 (6 at most)
    uint64_t w[12];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if ((uint32_t)k < nq) v = __ldg(q + k);
        w[2 * k] = ((uint64_t)v.y << 32) | v.x;
        w[2 * k + 1] = ((uint64_t)v.w << 32) | v.z;
    }
    const bool odd = skip >= 8;
    const uint32_t sh = (skip & 7) * 8;
    auto word = [&](int j) -> uint64_t {  // bytes [p + 8j, p + 8j + 8), little-endian
        const uint64_t lo = odd ? w[j + 1] : w[j];
        const uint64_t hi = (j + 2 < 12) ? (odd ? w[j + 2] : w[j + 1]) : 0ull;
        return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
    };
    auto tail8 = [&](uint64_t h, uint64_t x) -> uint64_t {
        h ^= round(0, x);
        return rotl(h, 27) * P1 + P4;
    };
    auto aval = [&](uint64_t h) -> uint64_t {
        h ^= h >> 33;
        h *= P2;
        h ^= h >> 29;
        h *= P3;
        h ^= h >> 32;
        return h;
    };
    auto merged = [&](uint64_t v1, uint64_t v2, uint64_t v3, uint64_t v4) -> uint64_t {
        uint64_t h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
        h = merge(h, v1);
        h = merge(h, v2);
        h = merge(h, v3);
        return merge(h, v4);
    };
    const uint64_t w0 = word(0);
    if (want & 1u) out[0] = filter_hash(aval(tail8(P5 + 8, w0)));
    if (len < 24) return;
    const uint64_t w1 = word(1), w2 = word(2);
    if (want & 2u) out[stride] = filter_hash(aval(tail8(tail8(tail8(P5 + 24, w0), w1), w2)));
    if (len < 40 || !(want & 12u)) return;
    uint64_t v1 = round(P1 + P2, w0), v2 = round(P2, w1), v3 = round(0, w2), v4 = round(0 - P1, word(3));
    if (want & 4u) out[2 * stride] = filter_hash(aval(tail8(merged(v1, v2, v3, v4) + 40, word(4))));
    if (len < 72 || !(want & 8u)) return;
    v1 = round(v1, word(4));
    v2 = round(v2, word(5));
    v3 = round(v3, word(6));
    v4 = round(v4, word(7));
    out[3 * stride] = filter_hash(aval(tail8(merged(v1, v2, v3, v4) + 72, word(8))));
}

// ------------------------------------------------------------ utilities ----
// Exclusive scan of u32 values; writes the total to *total (device).
// Scratch: scan_scratch_bytes(n).
uint64_t scan_scratch_bytes(uint64_t n);
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, void* scratch,
                       cudaStream_t st);
// Exclusive scan of u32 values into u64 sums (same scratch size).
int exclusive_scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, uint64_t* total, void* scratch,
                              cudaStream_t st);

inline unsigned grid_for(uint64_t n, unsigned block) {
    uint64_t g = (n + block - 1) / block;
    return (unsigned)(g ? g : 1);
}

}  // namespace dsss

struct dsss_ctx : dsss::Ctx {};
