// K3 — segmented MSD string sort with LCP output, the role radixsort_CI3
// plays per PE in the reference (tlx/sort/strings/radix_sort.hpp:861-884,
// called at src/sorter/distributed/prefix_doubling.hpp:228).
//
// Elements are string ids; every segment is sorted independently (a PE's
// strings, or the whole set).  Large segments (> small_max) are refined by
// MSD passes over 8-byte big-endian key chunks:
//   prefix   : common prefix of the segment (compare each string with the
//              first one), so a segment's key starts at its first differing byte;
//   keys/diff: gather the 8-byte key at that depth, OR of (key ^ key0) tells
//              which key byte is the first to differ;
//   hist     : warp-aggregated 256-bin histogram of that byte per 4096-element tile;
//   scan     : per segment, bucket starts and per-tile offsets (chunked);
//   scatter  : stable scatter of ids (and keys of children that stay large).
// A child that keeps more than half of its parent (a chain of long shared
// prefixes, e.g. suffixes inside repeats or strings that share a long common
// head) would lose one byte per pass; it is flagged for a pivot pass instead:
// every string's LCP with the segment's first string (up to 127 bytes) and
// the byte after it become a two-byte pseudo key whose order is the strings'
// order, so one pass resolves up to 127 bytes of the chain.
// Children of size <= small_max finish in one CTA (small_sort): bitonic sort
// of (group, key, id) in shared memory, tie groups re-keyed 8 bytes deeper
// until every group is a single string or byte-identical strings.
// LCPs are written where they become known: depth + first differing byte at
// every bucket / group boundary, the length for byte-identical neighbours.
// Ties between byte-identical strings keep ascending id order.
#include <algorithm>

#include "internal.cuh"
#include "strsort.cuh"

namespace dsss {

constexpr int LT_NT = 256, LT_IPT = 8, LT_TILE = LT_NT * LT_IPT;
constexpr int CHUNK_TILES = 32;
constexpr uint32_t PREFIX_CAP = 256;
// F_KEYS: the key array holds the segment's keys at Seg.depth; F_PIVOT: the
// next pass is a pivot pass; F_PSEUDO: the keys are pivot pseudo keys.
constexpr uint32_t F_PARITY = 1u, F_KEYS = 2u, F_PIVOT = 4u, F_PSEUDO = 8u;
constexpr uint32_t PIVOT_CAP = 127;  // pseudo key byte 0 holds codes 0 .. 2 * PIVOT_CAP

struct Seg {
    uint32_t start, size, depth, flags;
    uint32_t newdepth;
    uint32_t first_digit;
    unsigned long long diff;
    // speculated common-prefix depth + 1 (0: none) and the OR of key ^ key0
    // over the keys k_prefix wrote at that depth (segments without keys)
    uint32_t spec;
    // this pass's digit: the key byte at the first difference (nspl = 0), or
    // the bucket among nspl sampled splitters (table spl_slot; bucket-start
    // LCPs into the fix list from fix0)
    uint32_t nspl;
    unsigned long long spec_diff;
    uint32_t spl_slot, fix0;
    // OR and AND of the keys the previous pass's scatter wrote for this
    // segment (children with keys, when the child table is kept): the bits
    // that differ among its keys are kor ^ kand
    unsigned long long kor, kand;
};

// Sampled splitters.  Where the key byte at a large segment's first
// difference takes few values (letters, DNA), a byte digit splits the segment
// only a few ways per pass.  Instead, the distinct keys among every 8th of an
// evenly spaced, sorted sample of SPL_SAMPLE keys become m <= 255 splitters.
// With more than SPL_EQ_MAX of them a key's bucket is the number of
// splitters below it (about 1/256 of the segment each; two splitters are
// keys of the segment in different buckets, so it splits).  With fewer (few
// distinct keys: frequent ones), bucket 2j holds the keys between splitters
// j-1 and j and bucket 2j+1 the keys equal to splitter j, so every sampled
// key lands in an equality bucket and the others elsewhere.  Equal keys
// always share a bucket, and two neighbours across a bucket boundary have
// different keys, so their LCP is the depth plus the LCP of the two keys; it
// is written once the final order is known (k_lcp_fix).
constexpr int SPL_SAMPLE = 2048;
constexpr uint32_t SPL_MAX = 255, SPL_STRIDE = 256, SPL_EQ_MAX = 127;
constexpr uint32_t SPL_MIN_FLOOR = 4096;  // smallest sort_split_min other than 0 (off)
constexpr uint32_t FIX_NONE = 0xFFFFFFFFu;

constexpr int NBINS = 4;
__host__ __device__ constexpr int bin_cap(int b) { return b == 0 ? 32 : b == 1 ? 256 : b == 2 ? 1024 : 4096; }
__device__ __forceinline__ int bin_of(uint32_t size) {
    return size <= 32 ? 0 : size <= 256 ? 1 : size <= 1024 ? 2 : 3;
}

// Counters block (device): [0] n_large_next, [1..4] n_small per bin, [5]
// fix-list slots reserved, [6] splitter tables of the pass, [8] total tiles,
// [9] total chunks, [10] error flag (a guard tripped), [11] large segments of
// the next pass without keys or with a pivot pass.
struct SortState {
    ArenaDev a;
    uint32_t* ord[2];
    unsigned long long* key[2];
    uint32_t* ord_out;
    uint32_t* lcp_out;
    Seg* large[2];
    Seg* small[NBINS];
    uint32_t* tile0;
    uint32_t* chunk0;
    uint32_t* tmp_counts;
    uint32_t* tile_hist;
    uint32_t* chunk_pre;
    uint32_t* bucket;  // 257 per large segment
    uint32_t* counters;
    // child table (optional, 256 per large segment): the next list's slot of
    // digit d's child when it is large and keeps the keys (~0u otherwise); the
    // scatter then folds the keys it writes into that child's kor / kand
    uint32_t* child;
    Seg* nxt;  // the next pass's list (the scatter's children)
    uint32_t small_max;
    uint32_t pivot;  // pivot passes enabled
    uint32_t bits;   // plain keys split on their top differing bits: 0 never, 1 always, 2 on narrow bytes
    uint32_t seg_bits;  // the same inside the segment sorter
    uint32_t first;     // the first pass over the arena (host-driven passes)
    uint64_t cap_large, cap_small, cap_tiles, cap_chunks;
    // first pass only: every string's prefix hashes at the first schedule
    // depths (root_digests), ROOT_DIGESTS arrays of dig_n entries
    unsigned long long* dig;
    uint64_t dig_n;
    // sampled splitters: segments of at least split_min strings (0: never);
    // cap_spl tables of SPL_STRIDE keys per pass; the fix list holds
    // (position, depth) pairs of bucket starts whose LCP k_lcp_fix writes
    uint32_t split_min;
    const uint32_t* seg_depth;  // optional: each segment's shared prefix length
    unsigned long long* spl;
    uint32_t* fix;
    uint64_t cap_spl, cap_fix;
};

__device__ __forceinline__ uint32_t find_seg(const uint32_t* first, uint32_t nseg, uint32_t t) {
    // last s with first[s] <= t
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void push_small(const SortState& S, uint32_t start, uint32_t size, uint32_t depth,
                                           uint32_t flags) {
    int b = bin_of(size);
    uint32_t slot = atomicAdd(&S.counters[1 + b], 1u);
    if (slot >= S.cap_small) {
        atomicExch(&S.counters[10], 1u);
        return;
    }
    Seg s;
    s.start = start;
    s.size = size;
    s.depth = depth;
    s.flags = flags;
    s.newdepth = 0xFFFFFFFFu;
    s.first_digit = 0;
    s.diff = 0;
    s.spec = 0;
    s.nspl = 0;
    s.spl_slot = 0;
    s.fix0 = 0;
    s.spec_diff = 0;
    s.kor = 0;
    s.kand = ~0ull;
    S.small[b][slot] = s;
}

// Returns the segment's slot in dst (~0u when the list is full).
__device__ __forceinline__ uint32_t push_large(const SortState& S, Seg* dst, uint32_t start, uint32_t size,
                                               uint32_t depth, uint32_t flags) {
    uint32_t slot = atomicAdd(&S.counters[0], 1u);
    if (slot >= S.cap_large) {
        atomicExch(&S.counters[10], 1u);
        return 0xFFFFFFFFu;
    }
    if (!(flags & F_KEYS) || (flags & F_PIVOT)) atomicAdd(&S.counters[11], 1u);
    Seg s;
    s.start = start;
    s.size = size;
    s.depth = depth;
    s.flags = flags;
    s.newdepth = 0xFFFFFFFFu;
    s.first_digit = 0;
    s.diff = 0;
    s.spec = 0;
    s.nspl = 0;
    s.spl_slot = 0;
    s.fix0 = 0;
    s.spec_diff = 0;
    s.kor = 0;
    s.kand = ~0ull;
    dst[slot] = s;
    return slot;
}

// ------------------------------------------------------------------ init ----
__global__ void k_init_ids(uint32_t* ord, const uint32_t* in, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ord[i] = in ? in[i] : (uint32_t)i;
}

__global__ void k_init_segs(SortState S, const uint64_t* pb, uint32_t p) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p) return;
    uint32_t start = (uint32_t)pb[q], size = (uint32_t)(pb[q + 1] - pb[q]);
    if (size == 0) return;
    S.lcp_out[start] = 0;
    if (size == 1) {
        S.ord_out[start] = S.ord[0][start];
        return;
    }
    // a segment whose strings are known to share their first bytes starts there
    const uint32_t d = S.seg_depth ? S.seg_depth[q] : 0u;
    if (size > S.small_max) push_large(S, S.large[0], start, size, d, 0);
    else push_small(S, start, size, d, 0);
}

// --------------------------------------------------------- tile indexing ----
__global__ void k_tile_counts(const Seg* segs, uint32_t nseg, uint32_t* tiles, uint32_t* chunks) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    uint32_t t = (segs[s].size + LT_TILE - 1) / LT_TILE;
    tiles[s] = t;
    chunks[s] = (t + CHUNK_TILES - 1) / CHUNK_TILES;
}

// ---------------------------------------------------------------- prefix ----
// Big-endian key words [d, d + 8 W) of a string (0 past its end) from at most
// W + 1 aligned 8-byte loads, all issued before any is used.  Words wholly
// past the end are not loaded, so at most 15 bytes past a string are read
// (the arena contract pads 32).
template <int W>
__device__ __forceinline__ void key_words(const uint8_t* chars, uint64_t off, uint32_t len, uint32_t d,
                                          uint32_t want, uint64_t (&x)[W]) {
    const uint32_t avail = d < len ? (len - d + 7) >> 3 : 0;
    const uint32_t words = want < avail ? want : avail;
    const uintptr_t p = (uintptr_t)(chars + off + d);
    const unsigned long long* q = (const unsigned long long*)(p & ~(uintptr_t)7);
    const unsigned sh = (unsigned)(p & 7) * 8;
    uint64_t raw[W + 1];
    const uint32_t loads = words ? words + (sh != 0) : 0;
#pragma unroll
    for (int w = 0; w <= W; ++w) raw[w] = (uint32_t)w < loads ? __ldg(q + w) : 0ull;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        uint64_t v = sh ? (raw[w] >> sh) | (raw[w + 1] << (64 - sh)) : raw[w];
        const uint32_t at = d + 8 * w;
        if ((uint32_t)w >= words || at >= len) {
            v = 0;
        } else if (len - at < 8) {
            v &= (1ull << ((len - at) * 8)) - 1;
        }
        x[w] = bswap64(v);
    }
}

constexpr int PF_W = 8;  // prefix words compared per batch (64 bytes)
constexpr uint32_t SPEC_MAX = 56;  // speculated depths stay below d0 + 56 (key inside 64 bytes)

// Speculated common prefix of each segment without keys: the smallest LCP with
// the segment's first string over up to 256 evenly spaced members, when it is
// below d0 + SPEC_MAX.  k_prefix then reads each string once for both the
// check (the segment's common prefix is exactly that depth iff no member
// leaves the first string earlier) and the key at that depth; a wrong guess
// only costs the usual key gather of k_keys_diff.  Segments whose samples all
// share SPEC_MAX bytes keep the plain prefix search (long common prefixes).
__global__ void __launch_bounds__(256) k_spec(SortState S, Seg* segs, uint32_t nseg) {
    __shared__ uint32_t wmin[8];
    for (uint32_t si = blockIdx.x; si < nseg; si += gridDim.x) {
        Seg& sg = segs[si];
        if (sg.flags & (F_KEYS | F_PIVOT)) continue;  // the same for the whole block
        const uint32_t* ord = S.ord[sg.flags & F_PARITY];
        const uint32_t d0 = sg.depth;
        uint32_t l = 0xFFFFFFFFu;
        const uint32_t m = sg.size < 256u ? sg.size : 256u;
        if (threadIdx.x < m) {
            uint64_t off0, off;
            uint32_t len0, len;
            str_of(S.a, ord[sg.start], off0, len0);
            const uint32_t i = sg.start + (uint32_t)((uint64_t)threadIdx.x * sg.size / m);
            str_of(S.a, ord[i], off, len);
            uint64_t x[7], y[7];
            key_words<7>(S.a.chars, off, len, d0, 7, x);
            key_words<7>(S.a.chars, off0, len0, d0, 7, y);
            l = d0 + SPEC_MAX;
#pragma unroll
            for (int w = 6; w >= 0; --w) {  // the first word that differs or ends wins
                if (x[w] != y[w]) l = d0 + 8 * w + key_lcp(x[w], y[w]);
                else if (zero_byte(x[w]) < 8) l = d0 + 8 * w + zero_byte(x[w]);
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) l = min(l, __shfl_xor_sync(0xffffffffu, l, o));
        if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = l;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t v = wmin[0];
            for (int w = 1; w < 8; ++w) v = min(v, wmin[w]);
            sg.spec = v < d0 + SPEC_MAX ? v + 1 : 0u;
            sg.spec_diff = 0;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(LT_NT, 4) k_prefix(SortState S, Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    const uint32_t t = blockIdx.x;
    if (t >= S.counters[8]) return;
    const uint32_t si = find_seg(S.tile0, nseg, t);
    Seg& sg = segs[si];
    if (sg.flags & (F_KEYS | F_PIVOT)) return;
    const uint32_t par = sg.flags & F_PARITY;
    const uint32_t* ord = S.ord[par];
    const uint32_t tb = sg.start + (t - S.tile0[si]) * LT_TILE;
    const uint32_t te = min(sg.start + sg.size, tb + LT_TILE);
    const uint32_t d0 = sg.depth, cap = d0 + PREFIX_CAP;
    const uint32_t s0 = ord[sg.start];
    // prefix hashes (first pass only) at the schedule depths past the common
    // prefix this segment is expected to have: at or below it every string of
    // the segment shares its prefix with the others, so a round there hashes
    // one root per segment and never reads stored hashes; a depth skipped
    // here is marked so that the rounds hash it from the strings
    uint32_t dmask = 0;
    if (S.dig) {
        const uint32_t shared = sg.spec ? sg.spec - 1 : d0 + SPEC_MAX;
        for (int j = 0; j < ROOT_DIGESTS; ++j)
            if (root_digest_depth(j) > shared) dmask |= 1u << j;
        if (dmask != (1u << ROOT_DIGESTS) - 1 && threadIdx.x == 0) atomicOr(&S.counters[15], ~dmask & 15u);
    }
    uint64_t off0;
    uint32_t len0;
    str_of(S.a, s0, off0, len0);
    // the first string's first 64 bytes from d0, shared by the block
    __shared__ unsigned long long y[PF_W];
    if (threadIdx.x == 0) {
        uint64_t v[PF_W];
        key_words<PF_W>(S.a.chars, off0, len0, d0, PF_W, v);
#pragma unroll
        for (int w = 0; w < PF_W; ++w) y[w] = v[w];
    }
    __syncthreads();
    if (sg.spec) {
        // speculated depth D: LCP with the first string capped at D, and the
        // key at D, from one load of the words covering [d0, D + 8)
        const uint32_t D = sg.spec - 1, rel = D - d0;
        const uint32_t want = (rel + 15) >> 3;
        const uint32_t kw = rel >> 3, kr = (rel & 7) * 8;
        const uint64_t key0 = kr ? (y[kw] << kr) | (y[kw + 1] >> (64 - kr)) : y[kw];
        unsigned long long* key = S.key[par];
        uint32_t mn = 0xFFFFFFFFu;
        uint64_t df = 0;
        for (uint32_t i = tb + threadIdx.x; i < te; i += LT_NT) {
            uint64_t off;
            uint32_t len;
            const uint32_t s = ord[i];
            str_of(S.a, s, off, len);
            if (dmask) root_digests(S.a.chars + off, len, S.dig + s, S.dig_n, dmask);
            uint64_t x[PF_W];
            key_words<PF_W>(S.a.chars, off, len, d0, want, x);
            uint32_t l = D;
#pragma unroll
            for (int w = PF_W - 1; w >= 0; --w) {  // the first word that differs or ends wins
                if ((uint32_t)(8 * w) < rel) {
                    if (x[w] != y[w]) l = min(D, d0 + 8 * w + key_lcp(x[w], y[w]));
                    else if (zero_byte(x[w]) < 8) l = min(D, d0 + 8 * w + zero_byte(x[w]));
                }
            }
            uint64_t lo = 0, hi = 0;  // words kw and kw + 1, selected without indexing x at run time
#pragma unroll
            for (int w = 0; w < PF_W; ++w) {
                if ((uint32_t)w == kw) lo = x[w];
                if ((uint32_t)w == kw + 1) hi = x[w];
            }
            const uint64_t k = kr ? (lo << kr) | (hi >> (64 - kr)) : lo;
            key[i] = k;
            df |= k ^ key0;
            mn = min(mn, l);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            df |= __shfl_xor_sync(0xffffffffu, df, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (mn != 0xFFFFFFFFu) atomicMin(&sg.newdepth, mn);
            if (df) atomicOr(&sg.spec_diff, (unsigned long long)df);
        }
        return;
    }
    uint32_t mn = 0xFFFFFFFFu;
    for (uint32_t i = tb + threadIdx.x; i < te; i += LT_NT) {
        uint64_t off;
        uint32_t len;
        const uint32_t s = ord[i];
        str_of(S.a, s, off, len);
        if (dmask) root_digests(S.a.chars + off, len, S.dig + s, S.dig_n, dmask);
        // no need to compare past this thread's minimum so far
        const uint32_t lim = min(cap, mn);
        uint32_t l = 0;
        bool done = false;
        // first batch: every word up to the limit loaded at once
        {
            const uint32_t want = lim > d0 ? min((lim - d0 + 7) >> 3, (uint32_t)PF_W) : 0u;
            uint64_t x[PF_W];
            key_words<PF_W>(S.a.chars, off, len, d0, want, x);
#pragma unroll
            for (int w = 0; w < PF_W; ++w) {
                if (!done && (uint32_t)w < want) {
                    if (x[w] != y[w]) {
                        l = d0 + 8 * w + key_lcp(x[w], y[w]);
                        done = true;
                    } else {
                        const uint32_t z = zero_byte(x[w]);
                        if (z < 8) {
                            l = d0 + 8 * w + z;
                            done = true;
                        }
                    }
                }
            }
            if (!done && d0 + 8 * want >= lim) {
                l = d0 + 8 * want;
                done = true;
            }
        }
        // longer common prefixes: 16 bytes per step
        for (uint32_t d = d0 + 8 * PF_W; !done;) {
            uint64_t xx[2], yy[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                xx[q] = key8(S.a.chars, off, len, d + 8 * q);
                yy[q] = key8(S.a.chars, off0, len0, d + 8 * q);
            }
            l = d + 16;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!done) {
                    if (xx[q] != yy[q]) {
                        l = d + 8 * q + key_lcp(xx[q], yy[q]);
                        done = true;
                    } else {
                        const uint32_t z = zero_byte(xx[q]);
                        if (z < 8) {
                            l = d + 8 * q + z;
                            done = true;
                        }
                    }
                }
            }
            if (done) break;
            d += 16;
            if (d >= lim) {
                l = d;
                break;
            }
        }
        mn = min(mn, l);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if ((threadIdx.x & 31) == 0 && mn != 0xFFFFFFFFu) atomicMin(&sg.newdepth, mn);
}

// ------------------------------------------------------------- keys/diff ----
constexpr int KD_ILP = 8;
__global__ void __launch_bounds__(LT_NT) k_keys_diff(SortState S, Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    const uint32_t t = blockIdx.x;
    if (t >= S.counters[8]) return;
    const uint32_t si = find_seg(S.tile0, nseg, t);
    Seg& sg = segs[si];
    if (sg.flags & F_PIVOT) return;  // keys and diff come from k_pivot
    if (!(sg.flags & F_KEYS) && sg.spec && sg.newdepth == sg.spec - 1) {
        // the speculated depth was the common prefix: k_prefix wrote the keys
        if (t == S.tile0[si] && threadIdx.x == 0) sg.diff = sg.spec_diff;
        return;
    }
    const uint32_t par = sg.flags & F_PARITY;
    const bool valid = sg.flags & F_KEYS;
    const uint32_t depth = valid ? sg.depth : sg.newdepth;
    const uint32_t* ord = S.ord[par];
    unsigned long long* key = S.key[par];
    const uint32_t tb = sg.start + (t - S.tile0[si]) * LT_TILE;
    const uint32_t te = min(sg.start + sg.size, tb + LT_TILE);
    uint64_t k0;
    if (valid) {
        k0 = key[sg.start];
    } else {
        uint32_t s0 = ord[sg.start];
        k0 = key8_of(S.a, s0, depth);
    }
    uint64_t df = 0;
    if (valid) {
        // the tile's keys all in flight before any is used
        uint64_t k[LT_IPT];
#pragma unroll
        for (int j = 0; j < LT_IPT; ++j) {
            const uint32_t i = tb + j * LT_NT + threadIdx.x;
            k[j] = i < te ? key[i] : k0;
        }
#pragma unroll
        for (int j = 0; j < LT_IPT; ++j) df |= k[j] ^ k0;
    } else {
        // KD_ILP independent gathers in flight per thread
        for (uint32_t i0 = tb + threadIdx.x; i0 < te; i0 += KD_ILP * LT_NT) {
            uint32_t s[KD_ILP];
            uint64_t off[KD_ILP];
            uint32_t len[KD_ILP];
#pragma unroll
            for (int q = 0; q < KD_ILP; ++q) {
                const uint32_t i = i0 + q * LT_NT;
                s[q] = i < te ? ord[i] : 0u;
            }
#pragma unroll
            for (int q = 0; q < KD_ILP; ++q) {
                const uint32_t i = i0 + q * LT_NT;
                off[q] = 0;
                len[q] = 0;
                if (i < te) str_of(S.a, s[q], off[q], len[q]);
            }
#pragma unroll
            for (int q = 0; q < KD_ILP; ++q) {
                const uint32_t i = i0 + q * LT_NT;
                if (i < te) {
                    const uint64_t k = key8(S.a.chars, off[q], len[q], depth);
                    key[i] = k;
                    df |= k ^ k0;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) df |= __shfl_xor_sync(0xffffffffu, df, o);
    if ((threadIdx.x & 31) == 0 && df) atomicOr(&sg.diff, (unsigned long long)df);
}

// ------------------------------------------------------ sampled splitters ----
// Per large segment with keys (not a pivot pass) of at least split_min
// strings: the sample's byte-digit histogram at the first difference decides
// whether splitters pay (its largest bucket holds more than 1/64 of the
// sample, four times what a splitter bucket holds); if so, the sorted
// sample's every 8th key, distinct, become the splitters.  One block of
// SPL_SAMPLE / 2 threads per segment.
__global__ void __launch_bounds__(SPL_SAMPLE / 2) k_split_sample(SortState S, Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    __shared__ unsigned long long sk[SPL_SAMPLE];
    __shared__ uint32_t bcnt[256];
    __shared__ uint32_t s_fix0, s_nres;
    for (uint32_t si = blockIdx.x; si < nseg; si += gridDim.x) {
        Seg& sg = segs[si];
        const bool use = S.split_min && sg.size >= S.split_min && sg.diff != 0 && !(sg.flags & (F_PIVOT | F_PSEUDO));
        if (!use) {  // the same for the whole block
            if (threadIdx.x == 0) sg.nspl = 0;
            continue;
        }
        const unsigned long long* key = S.key[sg.flags & F_PARITY];
        const uint32_t shift = 56 - 8 * (uint32_t)(__clzll(sg.diff) >> 3);
        if (threadIdx.x < 256) bcnt[threadIdx.x] = 0;
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < (uint32_t)SPL_SAMPLE; j += blockDim.x) {
            const unsigned long long k = key[sg.start + (uint32_t)((uint64_t)j * sg.size / SPL_SAMPLE)];
            sk[j] = k;
            atomicAdd(&bcnt[(uint32_t)(k >> shift) & 0xFFu], 1u);
        }
        __syncthreads();
        // bitonic sort of the sample, ascending: thread t compares index i
        // (bit j clear) with i | j
        for (uint32_t k = 2; k <= (uint32_t)SPL_SAMPLE; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                const uint32_t i = ((threadIdx.x & ~(j - 1)) << 1) | (threadIdx.x & (j - 1));
                const unsigned long long a = sk[i], b = sk[i | j];
                if ((a > b) == ((i & k) == 0)) {
                    sk[i] = b;
                    sk[i | j] = a;
                }
                __syncthreads();
            }
        }
        if (threadIdx.x == 0) {
            uint32_t mx = 0;
            for (int d = 0; d < 256; ++d) mx = max(mx, bcnt[d]);
            uint32_t m = 0, slot = 0, fix0 = 0, nres = 0;
            if (64 * mx > (uint32_t)SPL_SAMPLE) {
                slot = atomicAdd(&S.counters[6], 1u);
                if (slot < S.cap_spl) {
                    unsigned long long* spl = S.spl + (uint64_t)slot * SPL_STRIDE;
                    for (uint32_t q = 0; q < SPL_MAX; ++q) {
                        const unsigned long long c = sk[(q + 1) * (SPL_SAMPLE / SPL_STRIDE) - 1];
                        if (m == 0 || c != spl[m - 1]) spl[m++] = c;
                    }
                    for (uint32_t q = m; q < SPL_STRIDE; ++q) spl[q] = ~0ull;
                    // bucket-start slots in the fix list, one per bucket
                    nres = m > SPL_EQ_MAX ? m + 1 : 2 * m + 1;
                    fix0 = atomicAdd(&S.counters[5], nres);
                    if ((uint64_t)fix0 + nres > S.cap_fix) m = 0;
                }
            }
            s_fix0 = fix0;
            s_nres = nres;
            sg.nspl = m;
            sg.spl_slot = slot;
            sg.fix0 = fix0;
        }
        __syncthreads();
        // every reserved fix slot starts empty (also a reservation past the
        // list's end, as far as the list goes)
        if (s_nres) {
            const uint64_t e = min((uint64_t)s_fix0 + s_nres, S.cap_fix);
            for (uint64_t f = (uint64_t)s_fix0 + threadIdx.x; f < e; f += blockDim.x) S.fix[2 * f] = FIX_NONE;
        }
        __syncthreads();  // the sample buffer is reused by the next segment
    }
}

// Bucket of key k among m sorted splitters (the table padded to SPL_STRIDE
// with ~0): j = the number of splitters below k (at most m, eight fixed
// steps); with more than SPL_EQ_MAX splitters j, else 2j, or 2j + 1 when k
// equals splitter j.
__device__ __forceinline__ uint32_t spl_bucket(const unsigned long long* spl, uint32_t m, unsigned long long k) {
    uint32_t j = 0;
#pragma unroll
    for (uint32_t step = SPL_STRIDE / 2; step; step >>= 1)
        if (spl[j + step - 1] < k) j += step;
    if (m > SPL_EQ_MAX) return j;
    return 2 * j + (j < m && spl[j] == k ? 1u : 0u);
}

// LCPs at the bucket starts of splitter passes, once the order is final: the
// two neighbours have different keys at depth d.
__global__ void __launch_bounds__(256) k_lcp_fix(SortState S) {
    const uint64_t m = min((uint64_t)S.counters[5], S.cap_fix);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; f < m; f += stride) {
        const uint32_t pos = S.fix[2 * f];
        if (pos == FIX_NONE) continue;
        uint32_t l = S.fix[2 * f + 1];
        const uint32_t x = S.ord_out[pos - 1], y = S.ord_out[pos];
        for (;;) {
            const uint64_t kx = key8_of(S.a, x, l), ky = key8_of(S.a, y, l);
            if (kx != ky) {
                l += key_lcp(kx, ky);
                break;
            }
            const uint32_t z = zero_byte(kx);
            if (z < 8) {
                l += z;
                break;
            }
            l += 8;
        }
        S.lcp_out[pos] = l;
    }
}

// ----------------------------------------------------------------- pivot ----
// Pivot pass of an F_PIVOT segment at depth d (all its strings share their
// first d bytes) with s0 its first string.  For string x, l = LCP(x, s0)
// counted from d and capped at PIVOT_CAP, and x's pseudo key holds
//   byte 0: code = l            if x < s0 (x's byte at l is smaller: x ends
//                               there or differs downwards),
//                = PIVOT_CAP    if x matches s0 for PIVOT_CAP bytes or equals it,
//                = 2*PIVOT_CAP - l  if x > s0;
//   byte 1: x's byte at d + l (0 for the code PIVOT_CAP).
// Ascending pseudo keys are ascending strings: two strings below s0 with
// different l compare at the smaller l, where the one with the smaller l has
// the smaller byte; above s0 the larger l comes first; equal codes compare by
// the byte at d + l.  Strings with the same pseudo key share their first
// d + l + 1 bytes (d + PIVOT_CAP for the middle code), and the LCP of two
// strings with different codes is d + min(l, l').
__device__ __forceinline__ uint32_t pivot_l(uint32_t code) { return code <= PIVOT_CAP ? code : 2 * PIVOT_CAP - code; }

// Pseudo key of string (off, len) against the pivot (off0, len0), both
// sharing their first d0 bytes.
__device__ __forceinline__ uint64_t pivot_key(const uint8_t* chars, uint64_t off, uint32_t len, uint64_t off0,
                                              uint32_t len0, uint32_t d0) {
    uint32_t code = PIVOT_CAP, byte = 0;
    bool done = false;
    for (uint32_t c = 0; c < PIVOT_CAP && !done; c += 16) {
        // 16 bytes per step: two independent 8-byte compares
        uint64_t x[2], y[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            x[q] = key8(chars, off, len, d0 + c + 8 * q);
            y[q] = key8(chars, off0, len0, d0 + c + 8 * q);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (done) continue;
            if (x[q] != y[q]) {
                const uint32_t j = key_lcp(x[q], y[q]);
                const uint32_t l = c + 8 * q + j;
                if (l < PIVOT_CAP) {
                    const uint32_t bx = (uint32_t)(x[q] >> (56 - 8 * j)) & 0xFFu;
                    const uint32_t by = (uint32_t)(y[q] >> (56 - 8 * j)) & 0xFFu;
                    code = bx < by ? l : 2 * PIVOT_CAP - l;
                    byte = bx;
                }
                done = true;
            } else if (zero_byte(x[q]) < 8) {
                done = true;  // equal to the pivot
            }
        }
    }
    return (uint64_t)code << 56 | (uint64_t)byte << 48;
}

__global__ void __launch_bounds__(LT_NT) k_pivot(SortState S, Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    const uint32_t t = blockIdx.x;
    if (t >= S.counters[8]) return;
    const uint32_t si = find_seg(S.tile0, nseg, t);
    Seg& sg = segs[si];
    if (!(sg.flags & F_PIVOT)) return;
    const uint32_t par = sg.flags & F_PARITY;
    const uint32_t* ord = S.ord[par];
    unsigned long long* key = S.key[par];
    const uint32_t tb = sg.start + (t - S.tile0[si]) * LT_TILE;
    const uint32_t te = min(sg.start + sg.size, tb + LT_TILE);
    uint64_t off0;
    uint32_t len0;
    str_of(S.a, ord[sg.start], off0, len0);
    const uint64_t k0 = (uint64_t)PIVOT_CAP << 56;
    uint64_t df = 0;
    for (uint32_t i = tb + threadIdx.x; i < te; i += LT_NT) {
        uint64_t off;
        uint32_t len;
        str_of(S.a, ord[i], off, len);
        const uint64_t k = pivot_key(S.a.chars, off, len, off0, len0, sg.depth);
        key[i] = k;
        df |= k ^ k0;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) df |= __shfl_xor_sync(0xffffffffu, df, o);
    if ((threadIdx.x & 31) == 0 && df) atomicOr(&sg.diff, (unsigned long long)df);
}

// ------------------------------------------------------------------ hist ----
__device__ __forceinline__ uint32_t digit_of(uint64_t k, uint32_t shift) { return (uint32_t)(k >> shift) & 0xFFu; }

// The digit of a pass over plain keys: the (up to) eight most significant
// bits in which the segment's keys differ, packed in key order.  Every bit
// above the lowest of them that is not one of them is the same in all keys,
// so the digit orders the keys as their first bytes do.  Where the key byte
// at the first difference varies in all eight bits this is that byte; over a
// small alphabet (letters vary in 5 or 6 bits of a byte, DNA in 4) a digit
// covers more than one key byte, and a pass splits up to 256 ways instead of
// as many ways as the byte has values.  sh[j]: the right shift that brings
// digit bit j (most significant first) to bit 0.
struct BitDigit {
    uint32_t nb;     // bits in the digit (1..8)
    uint32_t sh[8];
    bool whole;      // one whole key byte: (k >> sh[7]) & 0xFF
};

// Whether a pass over plain keys splits on bits: knob sort_bits 1 always, 2
// where the first differing key byte varies in at most four bits (DNA, or a
// leading digit with few values), 3 the same in the first pass only, 0
// never; and only for segments of more than four times the small-segment
// cutoff (a 256-way split of a segment just above the cutoff leaves children
// of a few strings each, whose segment records cost more than sorting them).
__device__ __forceinline__ bool use_bits(uint32_t mode, uint64_t diff, uint32_t shift, uint32_t size,
                                         uint32_t small_max, uint32_t first) {
    if ((uint64_t)size <= 4ull * small_max) return false;
    const bool narrow = __popc((uint32_t)(diff >> shift) & 0xFFu) <= 4;
    return mode == 1 || (mode == 2 && narrow) || (mode == 3 && first && narrow);
}

__device__ __forceinline__ BitDigit bit_digit_spec(uint64_t diff) {
    BitDigit d;
    d.nb = 0;
    uint64_t x = diff;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        d.sh[j] = 0;
        if (x) {
            const uint32_t at = 63u - (uint32_t)__clzll(x);
            d.sh[j] = at;
            x &= ~(1ull << at);
            ++d.nb;
        }
    }
    d.whole = d.nb == 8 && (d.sh[0] & 7u) == 7u && d.sh[7] + 7u == d.sh[0];
    return d;
}

// Digit lookup in shared memory: for each key byte that holds digit bits,
// tab[q][v] is the digit bits of byte value v, packed and moved to their place
// in the digit; a key's digit is the OR over those bytes (usually two).
struct BitTables {
    uint8_t tab[8][256];
    uint32_t n;      // key bytes holding digit bits
    uint32_t sh[8];  // right shift of each such byte
};

// Builds the tables of digit d; every thread of the block calls it, and a
// barrier follows before the first lookup.
__device__ __forceinline__ void bit_tables_build(BitTables& T, const BitDigit& d) {
    uint64_t chosen = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if ((uint32_t)j < d.nb) chosen |= 1ull << d.sh[j];
    for (uint32_t v = threadIdx.x; v < 256; v += blockDim.x) {
        uint32_t q = 0, below = (uint32_t)__popcll(chosen);
        for (int J = 0; J < 8; ++J) {
            const uint32_t sh = 56u - 8u * (uint32_t)J;
            const uint32_t sel = (uint32_t)(chosen >> sh) & 0xFFu;
            if (!sel) continue;
            below -= (uint32_t)__popc(sel);  // digit bits in later key bytes
            uint32_t x = 0;                  // the bits of v that sel selects, packed
            for (int bit = 7; bit >= 0; --bit)
                if ((sel >> bit) & 1u) x = (x << 1) | ((v >> bit) & 1u);
            T.tab[q][v] = (uint8_t)(x << below);
            if (v == 0) T.sh[q] = sh;
            ++q;
        }
        if (v == 0) T.n = q;
    }
}

__device__ __forceinline__ uint32_t bit_digit(uint64_t k, const BitDigit& d, const BitTables& T) {
    if (d.whole) return (uint32_t)(k >> d.sh[7]) & 0xFFu;
    uint32_t v = 0;
    for (uint32_t q = 0; q < T.n; ++q) v |= T.tab[q][(uint32_t)(k >> T.sh[q]) & 0xFFu];
    return v;
}

// Key byte (from the key's first byte) that holds digit bit h (0: least
// significant): two keys whose digits first differ in bit h share exactly
// that many bytes past the segment depth.
__device__ __forceinline__ uint32_t bit_digit_byte(const BitDigit& d, uint32_t h) {
    uint32_t byte = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if ((uint32_t)j + 1 + h == d.nb) byte = (63u - d.sh[j]) >> 3;
    return byte;
}

// BITS: the bit-digit form (its tables and registers only where the knob asks
// for it; the byte form keeps the occupancy of a 32-register kernel).
template <bool BITS>
__global__ void __launch_bounds__(LT_NT) k_hist(SortState S, const Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    // one 256-bin histogram per warp (shared-memory atomics contend only
    // inside a warp), summed per digit at the end
    __shared__ uint32_t hist[LT_NT / 32][256];
    __shared__ unsigned long long s_spl[SPL_STRIDE];
    const uint32_t t = blockIdx.x;
    if (t >= S.counters[8]) return;
    const uint32_t si = find_seg(S.tile0, nseg, t);
    const Seg sg = segs[si];
    if (sg.diff == 0) return;
    const uint32_t shift = 56 - 8 * (uint32_t)(__clzll(sg.diff) >> 3);
    const uint32_t m = sg.nspl;
    // plain keys split on their top differing bits, pivot pseudo keys on a byte
    const bool bits = BITS && !m && !(sg.flags & (F_PIVOT | F_PSEUDO)) && use_bits(S.bits, sg.diff, shift, sg.size, S.small_max, S.first);
    const BitDigit bd = bit_digit_spec(bits ? (uint64_t)sg.diff : (0xFFull << shift));
    __shared__ BitTables bt;
    if (BITS && !bd.whole) bit_tables_build(bt, bd);
    const unsigned long long* key = S.key[sg.flags & F_PARITY];
#pragma unroll
    for (int w = 0; w < LT_NT / 32; ++w) hist[w][threadIdx.x] = 0;
    if (m)
        for (uint32_t q = threadIdx.x; q < SPL_STRIDE; q += LT_NT) s_spl[q] = S.spl[(uint64_t)sg.spl_slot * SPL_STRIDE + q];
    __syncthreads();
    const uint32_t tb = sg.start + (t - S.tile0[si]) * LT_TILE;
    const uint32_t te = min(sg.start + sg.size, tb + LT_TILE);
    uint32_t* wh = hist[threadIdx.x >> 5];
    // the tile's keys loaded before any is counted (one DRAM wait, not LT_IPT)
    uint64_t k[LT_IPT];
#pragma unroll
    for (int j = 0; j < LT_IPT; ++j) {
        const uint32_t i = tb + j * LT_NT + threadIdx.x;
        k[j] = i < te ? key[i] : 0;
    }
#pragma unroll
    for (int j = 0; j < LT_IPT; ++j) {
        const uint32_t i = tb + j * LT_NT + threadIdx.x;
        if (i < te)
            atomicAdd(&wh[m ? spl_bucket(s_spl, m, k[j]) : BITS ? bit_digit(k[j], bd, bt) : digit_of(k[j], shift)], 1u);
    }
    __syncthreads();
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < LT_NT / 32; ++w) c += hist[w][threadIdx.x];
    S.tile_hist[(uint64_t)t * 256 + threadIdx.x] = c;
}

// ------------------------------------------------------------ chunk sums ----
__global__ void k_chunk_sum(SortState S, const Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    const uint32_t c = blockIdx.x;
    if (c >= S.counters[9]) return;
    const uint32_t si = find_seg(S.chunk0, nseg, c);
    const Seg sg = segs[si];
    if (sg.diff == 0) return;
    const uint32_t ntiles = (sg.size + LT_TILE - 1) / LT_TILE;
    const uint32_t t0 = S.tile0[si] + (c - S.chunk0[si]) * CHUNK_TILES;
    const uint32_t t1 = min(S.tile0[si] + ntiles, t0 + CHUNK_TILES);
    // each tile's count becomes its exclusive prefix inside the chunk (one
    // read for the scatter instead of the chunk's earlier tiles); every load
    // of the chunk in flight before the first store
    uint32_t v[CHUNK_TILES];
#pragma unroll
    for (int q = 0; q < CHUNK_TILES; ++q)
        v[q] = t0 + q < t1 ? S.tile_hist[(uint64_t)(t0 + q) * 256 + threadIdx.x] : 0u;
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < CHUNK_TILES; ++q) {
        if (t0 + q < t1) S.tile_hist[(uint64_t)(t0 + q) * 256 + threadIdx.x] = s;
        s += v[q];
    }
    S.chunk_pre[(uint64_t)c * 256 + threadIdx.x] = s;
}

// ----------------------------------------------------------- segment scan ----
__global__ void __launch_bounds__(256) k_seg_scan(SortState S, Seg* segs, uint32_t nseg, Seg* next) {
    __shared__ uint32_t sh[32];
    __shared__ uint32_t s_first;
    if (!segs) {  // graph mode: this pass's list and count live on the device
        const uint32_t c = S.counters[12];
        segs = S.large[c];
        next = S.large[c ^ 1u];
        nseg = S.counters[13];
    }
    const uint32_t si = blockIdx.x;
    if (si >= nseg) return;
    Seg& sg = segs[si];
    const uint32_t par = sg.flags & F_PARITY;
    const bool pseudo = (sg.flags & (F_PIVOT | F_PSEUDO)) != 0;
    const uint32_t depth = (sg.flags & (F_KEYS | F_PIVOT)) ? sg.depth : sg.newdepth;
    const uint32_t d = threadIdx.x;
    if (sg.diff == 0) {
        // Every key equal: byte-identical strings if the key holds their end,
        // else continue deeper without keys.
        const uint64_t k0 = S.key[par][sg.start];
        const uint32_t* ord = S.ord[par];
        uint32_t fin = 0xFFFFFFFFu, cont = 0, cflags = par;
        if (pseudo) {
            const uint32_t code = (uint32_t)(k0 >> 56), byte = (uint32_t)(k0 >> 48) & 0xFFu;
            if (code == PIVOT_CAP) {
                uint64_t o0;
                uint32_t l0;
                str_of(S.a, ord[sg.start], o0, l0);
                if (l0 < depth + PIVOT_CAP) fin = l0;  // all equal the pivot
                else cont = depth + PIVOT_CAP;
            } else if (byte == 0) {
                fin = depth + pivot_l(code);  // all end where they leave the pivot
            } else {
                cont = depth + pivot_l(code) + 1;
            }
            cflags |= F_PIVOT;
        } else {
            const uint32_t z = zero_byte(k0);
            if (z < 8) fin = depth + z;
            else cont = depth + 8;
        }
        if (fin != 0xFFFFFFFFu) {
            for (uint32_t i = threadIdx.x; i < sg.size; i += blockDim.x) {
                S.ord_out[sg.start + i] = ord[sg.start + i];
                if (i) S.lcp_out[sg.start + i] = fin;
            }
        } else if (threadIdx.x == 0) {
            push_large(S, next, sg.start, sg.size, cont, cflags);
        }
        return;
    }
    const uint32_t b = (uint32_t)(__clzll(sg.diff) >> 3);
    const uint32_t c0 = S.chunk0[si];
    const uint32_t ntiles = (sg.size + LT_TILE - 1) / LT_TILE;
    const uint32_t nch = (ntiles + CHUNK_TILES - 1) / CHUNK_TILES;
    // the digit's column of chunk sums, eight loads in flight (a segment of
    // n strings has n / 64 Ki chunks, walked by one block)
    uint32_t run = 0;
    for (uint32_t c = 0; c < nch; c += 8) {
        uint32_t v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = c + q < nch ? S.chunk_pre[(uint64_t)(c0 + c + q) * 256 + d] : 0u;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (c + q < nch) S.chunk_pre[(uint64_t)(c0 + c + q) * 256 + d] = run;
            run += v[q];
        }
    }
    const uint32_t total = run;
    // block exclusive scan over the 256 digits
    const int lane = d & 31, w = d >> 5;
    uint32_t x = total;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    if (d == 0) s_first = 256;
    __syncthreads();
    uint32_t wb = 0;
    for (int k = 0; k < w; ++k) wb += sh[k];
    const uint32_t excl = wb + x - total;
    if (total) atomicMin(&s_first, d);
    uint32_t* bk = S.bucket + (uint64_t)si * 257;
    bk[d] = sg.start + excl;
    if (d == 255) bk[256] = sg.start + sg.size;
    __syncthreads();
    if (d == 0) {
        sg.first_digit = s_first;
        sg.depth = depth;
    }
    uint32_t* child = S.child ? S.child + (uint64_t)si * 256 + d : nullptr;
    if (child) *child = 0xFFFFFFFFu;  // set below for a large child that keeps the keys
    if (total < 2) return;
    const uint32_t cs = sg.start + excl;
    const uint32_t np = par ^ 1u;
    if (sg.nspl) {
        // splitter buckets: children keep the keys at this depth (an
        // equality bucket's keys are all equal: its next pass goes deeper)
        if (total > S.small_max) {
            const uint32_t slot = push_large(S, next, cs, total, depth, np | F_KEYS);
            if (child) *child = slot;
        } else {
            push_small(S, cs, total, depth, np | F_KEYS);
        }
    } else if (!pseudo) {
        // digit 0 holds the strings that end at byte b, unless byte b has a
        // constant nonzero part (then no string ends there and digit 0 is an
        // ordinary bucket)
        bool ended_ok = true;
        if (S.bits) {
            const uint32_t shift = 56 - 8 * b;
            const uint64_t k0 = S.key[par][sg.start];
            ended_ok = (((k0 >> shift) & 0xFFu) & ~((sg.diff >> shift) & 0xFFu)) == 0;
        }
        if (d == 0 && ended_ok) return;  // strings that end here: written by the scatter
        // children keep the parent's keys: their first b+1 key bytes are now
        // common; one that keeps most of the parent gets a pivot pass
        if (total > S.small_max) {
            if (S.pivot && 2 * (uint64_t)total > sg.size) {
                push_large(S, next, cs, total, depth + b + 1, np | F_PIVOT);
            } else {
                const uint32_t slot = push_large(S, next, cs, total, depth, np | F_KEYS);
                if (child) *child = slot;
            }
        } else {
            push_small(S, cs, total, depth, np | F_KEYS);
        }
    } else if (b == 0) {
        // split by pivot code (only the pivot pass's own segment, whose first
        // string is the pivot): large children keep the pseudo keys, small
        // ones restart from the depth their strings share
        if (total > S.small_max) {
            const uint32_t slot = push_large(S, next, cs, total, depth, np | F_KEYS | F_PSEUDO);
            if (child) *child = slot;
        } else {
            uint32_t cd = depth + pivot_l(d);
            if (d == PIVOT_CAP) {
                uint64_t o0;
                uint32_t l0;
                str_of(S.a, S.ord[par][sg.start], o0, l0);
                cd = min(depth + PIVOT_CAP, l0);
            }
            push_small(S, cs, total, cd, np);
        }
    } else {
        // split by the byte after the shared d + l bytes; byte 0: strings that
        // end there, written by the scatter
        if (d == 0) return;
        const uint32_t cd = depth + pivot_l((uint32_t)(S.key[par][sg.start] >> 56)) + 1;
        if (total > S.small_max) push_large(S, next, cs, total, cd, np | (S.pivot && 2 * (uint64_t)total > sg.size ? F_PIVOT : 0u));
        else push_small(S, cs, total, cd, np);
    }
}

// --------------------------------------------------------------- scatter ----
// Ranks are stable within the tile (warp-aggregated per digit); the tile is
// first reordered by digit in shared memory so that the global writes of each
// digit's run are contiguous.
constexpr size_t SCATTER_SMEM = (size_t)LT_TILE * (8 + 4 + 1);

__global__ void __launch_bounds__(LT_NT, 4) k_scatter(SortState S, const Seg* segs, uint32_t nseg) {
    if (!segs) {  // graph mode: this pass's list and count live on the device
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    extern __shared__ __align__(16) unsigned char sm_scatter[];
    unsigned long long* skey = (unsigned long long*)sm_scatter;
    uint32_t* sord = (uint32_t*)(skey + LT_TILE);
    uint8_t* sdig = (uint8_t*)(sord + LT_TILE);
    __shared__ uint32_t base[256];
    __shared__ uint32_t bstart[257];
    __shared__ uint32_t tloff[256];
    __shared__ uint32_t wcnt[LT_NT / 32][256];
    __shared__ uint32_t wsum[LT_NT / 32];
    __shared__ uint32_t schild[256];
    __shared__ uint32_t actm[LT_NT / 32];  // per warp: the digits (d & 7 == warp) whose keys it folds
    __shared__ unsigned long long s_spl[SPL_STRIDE];
    const uint32_t t = blockIdx.x;
    if (t >= S.counters[8]) return;
    const uint32_t si = find_seg(S.tile0, nseg, t);
    const Seg sg = segs[si];
    if (sg.diff == 0) return;
    const uint32_t par = sg.flags & F_PARITY;
    const uint32_t b = (uint32_t)(__clzll(sg.diff) >> 3);
    const uint32_t shift = 56 - 8 * b;
    const uint32_t depth = sg.depth;
    const uint32_t m = sg.nspl;  // splitter buckets (0: the byte digit)
    const bool pseudo = (sg.flags & (F_PIVOT | F_PSEUDO)) != 0;
    // plain keys split on their top differing bits, pivot pseudo keys on a byte
    const bool bits = S.bits && !m && !pseudo && use_bits(S.bits, sg.diff, shift, sg.size, S.small_max, S.first);
    const BitDigit bd = bit_digit_spec(bits ? (uint64_t)sg.diff : (0xFFull << shift));
    __shared__ BitTables bt;
    if (!bd.whole) bit_tables_build(bt, bd);  // the barrier after the block's set-up follows
    // digit 0 holds the strings that end at byte b unless byte b has a
    // constant nonzero part
    bool ended_ok = true;
    if (bits) {
        const uint64_t k0 = S.key[par][sg.start];
        ended_ok = (((k0 >> shift) & 0xFFu) & ~((sg.diff >> shift) & 0xFFu)) == 0;
    }
    // LCP inside the group of strings that end here and at bucket starts
    // (pivot code splits: d + min(l, l') from the two codes)
    const bool code_split = pseudo && b == 0;
    const uint32_t lcp_here = pseudo ? depth + pivot_l((uint32_t)(S.key[par][sg.start] >> 56)) : depth + b;
    const uint32_t tloc = t - S.tile0[si];
    const uint32_t c = S.chunk0[si] + tloc / CHUNK_TILES;
    {
        const uint32_t d = threadIdx.x;
        const uint32_t* bk = S.bucket + (uint64_t)si * 257;
        // k_chunk_sum left the tile's prefix inside its chunk in tile_hist
        base[d] = bk[d] + S.chunk_pre[(uint64_t)c * 256 + d] + S.tile_hist[(uint64_t)t * 256 + d];
        bstart[d] = bk[d];
        if (d == 0) bstart[256] = bk[256];
        if (S.child) schild[d] = S.child[(uint64_t)si * 256 + d];
        if (d < LT_NT / 32) actm[d] = 0;
#pragma unroll
        for (int w = 0; w < LT_NT / 32; ++w) wcnt[w][d] = 0;
        if (m)
            for (uint32_t q = d; q < SPL_STRIDE; q += LT_NT) s_spl[q] = S.spl[(uint64_t)sg.spl_slot * SPL_STRIDE + q];
    }
    __syncthreads();
    const uint32_t* ord = S.ord[par];
    const unsigned long long* key = S.key[par];
    uint32_t* ord_dst = S.ord[par ^ 1u];
    unsigned long long* key_dst = S.key[par ^ 1u];
    const uint32_t tb = sg.start + tloc * LT_TILE;
    const uint32_t te = min(sg.start + sg.size, tb + LT_TILE);
    const uint32_t tn = te - tb;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t wb = tb + (uint32_t)w * 32 * LT_IPT;
    uint64_t k[LT_IPT];
    uint32_t o[LT_IPT];
    uint32_t rk[LT_IPT];
#pragma unroll
    for (int j = 0; j < LT_IPT; ++j) {
        const uint32_t i = wb + j * 32 + lane;
        k[j] = i < te ? key[i] : 0;
        o[j] = i < te ? ord[i] : 0;
    }
#pragma unroll
    for (int j = 0; j < LT_IPT; ++j) {
        const uint32_t i = wb + j * 32 + lane;
        const uint32_t dg = i < te ? (m ? spl_bucket(s_spl, m, k[j]) : bit_digit(k[j], bd, bt)) : 0x100u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, dg);
        const uint32_t r = __popc(peers & ((1u << lane) - 1));
        const uint32_t prev = dg < 256 ? wcnt[w][dg] : 0;
        __syncwarp();
        if (dg < 256 && lane == __ffs(peers) - 1) wcnt[w][dg] = prev + __popc(peers);
        __syncwarp();
        rk[j] = (dg & 0xFFu) << 24 | (prev + r);  // the digit kept for the placement below
    }
    __syncthreads();
    {
        // exclusive over warps per digit, then over digits within the tile
        const uint32_t d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < LT_NT / 32; ++ww) {
            const uint32_t v = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += v;
        }
        uint32_t x = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        uint32_t wpre = 0;
        for (int ww = 0; ww < w; ++ww) wpre += wsum[ww];
        tloff[d] = wpre + x - run;
        if (S.child && run && schild[d] < S.cap_large) atomicOr(&actm[d & 7], 1u << (d >> 3));
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < LT_IPT; ++j) {
        const uint32_t i = wb + j * 32 + lane;
        if (i >= te) continue;
        const uint32_t dg = rk[j] >> 24;
        const uint32_t lp = tloff[dg] + wcnt[w][dg] + (rk[j] & 0xFFFFFFu);
        if (lp >= tn) {  // never taken when the counts agree
            atomicExch(&S.counters[10], 1u);
            continue;
        }
        skey[lp] = k[j];
        sord[lp] = o[j];
        sdig[lp] = (uint8_t)dg;
    }
    __syncthreads();
    if (S.child) {
        // the OR and AND of the keys each large child that keeps them gets
        // from this tile (one warp per digit, over the digit's run in shared
        // memory): its next pass needs no key read to find the byte where its
        // keys differ
        for (uint32_t m = actm[w]; m; m &= m - 1) {
            const uint32_t dg = ((uint32_t)(__ffs(m) - 1) << 3) | (uint32_t)w;
            const uint32_t r0 = tloff[dg], r1 = dg < 255 ? tloff[dg + 1] : tn;
            unsigned long long vo = 0, va = ~0ull;
            for (uint32_t x = r0 + lane; x < r1; x += 32) {
                const unsigned long long v = skey[x];
                vo |= v;
                va &= v;
            }
            const uint32_t olo = __reduce_or_sync(0xffffffffu, (uint32_t)vo);
            const uint32_t ohi = __reduce_or_sync(0xffffffffu, (uint32_t)(vo >> 32));
            const uint32_t alo = __reduce_and_sync(0xffffffffu, (uint32_t)va);
            const uint32_t ahi = __reduce_and_sync(0xffffffffu, (uint32_t)(va >> 32));
            if (lane == 0) {
                const uint32_t slot = schild[dg];
                atomicOr(&S.nxt[slot].kor, ((unsigned long long)ohi << 32) | olo);
                atomicAnd(&S.nxt[slot].kand, ((unsigned long long)ahi << 32) | alo);
            }
        }
    }
    for (uint32_t x = threadIdx.x; x < tn; x += LT_NT) {
        const uint32_t dg = sdig[x];
        const uint32_t dest = base[dg] + (x - tloff[dg]);
        const uint32_t bs = bstart[dg], cnt = bstart[dg + 1] - bs;
        if (dest < bs || dest >= bs + cnt) {  // never taken when the counts agree
            atomicExch(&S.counters[10], 1u);
            continue;
        }
        const uint32_t oo = sord[x];
        const bool ended = !m && dg == 0 && !code_split && ended_ok;
        if (ended || cnt == 1) {
            S.ord_out[dest] = oo;
            if (ended && dest != bs) S.lcp_out[dest] = lcp_here;
        } else {
            ord_dst[dest] = oo;
            key_dst[dest] = skey[x];
        }
        if (m) {
            // a splitter bucket's start: its LCP once the order is final
            if (dest == bs && dg != sg.first_digit) {
                S.fix[2 * ((uint64_t)sg.fix0 + dg)] = dest;
                S.fix[2 * ((uint64_t)sg.fix0 + dg) + 1] = depth;
            }
        } else if (dest == bs && dg != sg.first_digit) {
            uint32_t l = lcp_here;
            if (code_split || !bd.whole) {
                uint32_t pd = dg - 1;  // previous non-empty bucket (exists: dg is not the first)
                while (pd > 0 && bstart[pd] == bs) --pd;
                // pivot codes: d + min(l, l'); bit digits: the byte of the
                // highest bit in which the two buckets' digits differ
                l = code_split ? depth + min(pivot_l(dg), pivot_l(pd))
                               : depth + bit_digit_byte(bd, 31u - (uint32_t)__clz(dg ^ pd));
            }
            S.lcp_out[dest] = l;
        }
    }
}

// ------------------------------------------------------------ small sort ----
// Segments of 2..small_max strings finish inside one CTA (the tail the MSD
// passes hand over, like the reference's insertion-sort / multikey tail):
//  - buckets of up to 32 strings, and of up to 64 from a wide split in the
//    large variants: one warp, a bitonic network across the 32 lanes (two
//    elements per lane above 32) on (group, key, id); groups of
//    equal keys jump to the depth where a member leaves the group's head and
//    are sorted again until each group is one string or byte-identical strings;
//  - larger buckets: an MSD pass in shared memory on the first key byte that
//    differs inside the bucket (warp-aggregated histogram, scan, stable
//    scatter); children go on a shared-memory stack or to the warp list.
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ bool lt3(uint32_t g1, uint64_t k1, uint32_t o1, uint32_t g2, uint64_t k2, uint32_t o2) {
    return g1 < g2 || (g1 == g2 && (k1 < k2 || (k1 == k2 && o1 < o2)));
}

// Lane i < size holds (key at `depth`, id).  On return lane i holds the i-th
// smallest; lcp[lane] (lanes 1..size-1) gets the LCP with the predecessor.
__device__ __forceinline__ void warp_sort(const ArenaDev& a, uint32_t size, uint32_t depth, uint64_t& key,
                                          uint32_t& id, uint32_t* lcp) {
    const int lane = threadIdx.x & 31;
    const bool valid = (uint32_t)lane < size;
    uint32_t grp = valid ? 0u : 0xFFFFFFFFu;
    uint32_t dep = depth;
    if (!valid) {
        key = ~0ull;
        id = 0xFFFFFFFFu;
    }
    for (bool first = true;; first = false) {
        if (first) {
            // one group at one depth (invalid lanes carry the largest key
            // and id, so they still sort last): (key, id) is the whole order
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint64_t pk = __shfl_xor_sync(FULL, key, j);
                    const uint32_t po = __shfl_xor_sync(FULL, id, j);
                    const bool want_min = ((lane & k) == 0) == ((lane & j) == 0);
                    const bool less = pk < key || (pk == key && po < id);
                    if (less == want_min) {
                        key = pk;
                        id = po;
                    }
                }
            }
        } else {
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint32_t pg = __shfl_xor_sync(FULL, grp, j);
                    const uint64_t pk = __shfl_xor_sync(FULL, key, j);
                    const uint32_t po = __shfl_xor_sync(FULL, id, j);
                    const uint32_t pd = __shfl_xor_sync(FULL, dep, j);
                    const bool want_min = ((lane & k) == 0) == ((lane & j) == 0);
                    const bool take = want_min ? lt3(pg, pk, po, grp, key, id) : lt3(grp, key, id, pg, pk, po);
                    if (take) {
                        grp = pg;
                        key = pk;
                        id = po;
                        dep = pd;
                    }
                }
            }
        }
        const uint32_t qg = __shfl_up_sync(FULL, grp, 1);
        const uint64_t qk = __shfl_up_sync(FULL, key, 1);
        const bool head = lane == 0 || qg != grp || qk != key;
        if (valid && lane > 0 && qg == grp) {
            if (qk != key) {
                lcp[lane] = dep + key_lcp(key, qk);
            } else {
                const uint32_t z = zero_byte(key);
                if (z < 8) lcp[lane] = dep + z;  // byte-identical neighbours
            }
        }
        const uint32_t heads = __ballot_sync(FULL, head);
        const uint32_t rs = 31u - __clz(heads & ((2u << lane) - 1u));
        const bool next_head = lane == 31 ? true : ((heads >> (lane + 1)) & 1u) != 0;
        const bool multi = !head || (!next_head && (uint32_t)(lane + 1) < size);
        const bool unres = valid && multi && zero_byte(key) == 8;
        if (valid) grp = rs;
        if (!__any_sync(FULL, unres)) break;
        // Every unresolved run shares its 8-byte key: jump to the first depth
        // where a member differs from the run head (or ends), the minimum over
        // the run of each member's LCP with the head.
        const uint32_t hid = __shfl_sync(FULL, id, rs);
        uint32_t l = 0xFFFFFFFFu;
        if (unres && (uint32_t)lane != rs) {
            uint64_t off, offh;
            uint32_t len, lenh;
            str_of(a, id, off, len);
            str_of(a, hid, offh, lenh);
            for (uint32_t d = dep + 8;; d += 16) {
                const uint64_t x0 = key8(a.chars, off, len, d), y0 = key8(a.chars, offh, lenh, d);
                const uint64_t x1 = key8(a.chars, off, len, d + 8), y1 = key8(a.chars, offh, lenh, d + 8);
                if (x0 != y0) { l = d + key_lcp(x0, y0); break; }
                if (zero_byte(x0) < 8) { l = d + zero_byte(x0); break; }
                if (x1 != y1) { l = d + 8 + key_lcp(x1, y1); break; }
                if (zero_byte(x1) < 8) { l = d + 8 + zero_byte(x1); break; }
            }
        }
        const uint32_t run = __match_any_sync(FULL, unres ? rs : 32u + (uint32_t)lane);
        const uint32_t nd = __reduce_min_sync(run, l);
        if (unres) {
            dep = nd;
            key = key8_of(a, id, dep);
        }
    }
}

// A bucket of at most T strings whose keys are in shared memory, sorted by
// one thread: an odd-even transposition network on (key, id) in registers
// (absent slots carry the largest pair, so they sort last), then the LCPs of
// neighbours.  Returns false,
// writing nothing, when two keys are equal and neither string ends inside
// them (a warp sort then goes deeper).
template <int T>
__device__ __forceinline__ bool tiny_sort(const unsigned long long* sk, uint32_t* so, uint32_t* lcp, uint32_t ws,
                                          uint32_t wn, uint32_t wd) {
    uint64_t k[T];
    uint32_t o[T];
#pragma unroll
    for (int i = 0; i < T; ++i) {
        o[i] = 0xFFFFFFFFu;
        k[i] = ~0ull;
        if ((uint32_t)i < wn) {
            o[i] = so[ws + i];
            k[i] = sk[ws + i];
        }
    }
#pragma unroll
    for (int pass = 0; pass < T; ++pass) {
#pragma unroll
        for (int i = pass & 1; i + 1 < T; i += 2) {
            if (k[i + 1] < k[i] || (k[i + 1] == k[i] && o[i + 1] < o[i])) {
                const uint64_t tk = k[i];
                k[i] = k[i + 1];
                k[i + 1] = tk;
                const uint32_t to = o[i];
                o[i] = o[i + 1];
                o[i + 1] = to;
            }
        }
    }
    bool ok = true;
#pragma unroll
    for (int i = 1; i < T; ++i)
        if ((uint32_t)i < wn && k[i - 1] == k[i] && zero_byte(k[i]) == 8) ok = false;
    if (!ok) return false;
#pragma unroll
    for (int i = 0; i < T; ++i) {
        if ((uint32_t)i < wn) {
            so[ws + i] = o[i];
            if (i) lcp[ws + i] = k[i - 1] != k[i] ? wd + key_lcp(k[i - 1], k[i]) : wd + zero_byte(k[i]);
        }
    }
    return true;
}

constexpr uint32_t WL_DONE = 1u << 31;  // warp-list entry finished by one thread
constexpr uint32_t TINY_MAX = 8;       // largest bucket one thread sorts

// Buckets of 33..64 strings: lane l holds positions l and l + 32 (elements 0
// and 1).  The same bitonic order on (group, key, id) over 64 positions (the
// stage j = 32 compares a lane's two elements), the same run handling as
// warp_sort; the run minima go through `scratch` (>= size words of shared
// memory owned by this warp).
__device__ __forceinline__ void cx_key_id(uint64_t& key, uint32_t& id, int j, bool want_min) {
    const uint64_t pk = __shfl_xor_sync(FULL, key, j);
    const uint32_t po = __shfl_xor_sync(FULL, id, j);
    const bool less = pk < key || (pk == key && po < id);
    if (less == want_min) {
        key = pk;
        id = po;
    }
}

__device__ __forceinline__ void cx_full(uint32_t& grp, uint64_t& key, uint32_t& id, uint32_t& dep, int j,
                                        bool want_min) {
    const uint32_t pg = __shfl_xor_sync(FULL, grp, j);
    const uint64_t pk = __shfl_xor_sync(FULL, key, j);
    const uint32_t po = __shfl_xor_sync(FULL, id, j);
    const uint32_t pd = __shfl_xor_sync(FULL, dep, j);
    const bool take = want_min ? lt3(pg, pk, po, grp, key, id) : lt3(grp, key, id, pg, pk, po);
    if (take) {
        grp = pg;
        key = pk;
        id = po;
        dep = pd;
    }
}

__device__ void warp_sort64(const ArenaDev& a, uint32_t size, uint32_t depth, uint64_t (&key)[2], uint32_t (&id)[2],
                            uint32_t* lcp, uint32_t* scratch) {
    const uint32_t lane = threadIdx.x & 31;
    bool valid[2];
    uint32_t grp[2], dep[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        valid[h] = lane + 32 * h < size;
        grp[h] = valid[h] ? 0u : 0xFFFFFFFFu;
        dep[h] = depth;
        if (!valid[h]) {
            key[h] = ~0ull;
            id[h] = 0xFFFFFFFFu;
        }
    }
    for (bool first = true;; first = false) {
#pragma unroll
        for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                if (j == 32) {  // k == 64: ascending, element 0 takes the smaller
                    // In the first network the group marks positions (valid
                    // or padding) and the depth is uniform: only (key, id)
                    // move, as in cx_key_id.
                    const bool sw = first ? (key[1] < key[0] || (key[1] == key[0] && id[1] < id[0]))
                                          : lt3(grp[1], key[1], id[1], grp[0], key[0], id[0]);
                    if (sw) {
                        uint64_t tk = key[0];
                        key[0] = key[1];
                        key[1] = tk;
                        uint32_t t = id[0];
                        id[0] = id[1];
                        id[1] = t;
                        if (!first) {
                            t = grp[0];
                            grp[0] = grp[1];
                            grp[1] = t;
                            t = dep[0];
                            dep[0] = dep[1];
                            dep[1] = t;
                        }
                    }
                    continue;
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t pos = lane + 32 * h;
                    const bool want_min = ((pos & k) == 0) == ((pos & j) == 0);
                    if (first) cx_key_id(key[h], id[h], j, want_min);
                    else cx_full(grp[h], key[h], id[h], dep[h], j, want_min);
                }
            }
        }
        // predecessor of each position: lane - 1 of the same half, lane 31 of
        // half 0 for position 32
        const uint64_t k31 = __shfl_sync(FULL, key[0], 31);
        const uint32_t g31 = __shfl_sync(FULL, grp[0], 31);
        bool head[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint64_t qu = __shfl_up_sync(FULL, key[h], 1);
            const uint32_t gu = __shfl_up_sync(FULL, grp[h], 1);
            const uint64_t qk = lane == 0 ? k31 : qu;
            const uint32_t qg = lane == 0 ? g31 : gu;
            const bool has_pred = h == 1 || lane > 0;
            head[h] = !has_pred || qg != grp[h] || qk != key[h];
            if (valid[h] && has_pred && qg == grp[h]) {
                const uint32_t pos = lane + 32 * h;
                if (qk != key[h]) {
                    lcp[pos] = dep[h] + key_lcp(key[h], qk);
                } else {
                    const uint32_t z = zero_byte(key[h]);
                    if (z < 8) lcp[pos] = dep[h] + z;  // byte-identical neighbours
                }
            }
        }
        const uint64_t heads = (uint64_t)__ballot_sync(FULL, head[0]) | (uint64_t)__ballot_sync(FULL, head[1]) << 32;
        bool unres[2];
        uint32_t rs[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t pos = lane + 32 * h;
            rs[h] = 63u - (uint32_t)__clzll(heads & ((2ull << pos) - 1ull));
            const bool next_head = pos == 63 ? true : ((heads >> (pos + 1)) & 1ull) != 0;
            const bool multi = !head[h] || (!next_head && pos + 1 < size);
            unres[h] = valid[h] && multi && zero_byte(key[h]) == 8;
            if (valid[h]) grp[h] = rs[h];
        }
        if (!__any_sync(FULL, unres[0] || unres[1])) break;
        // Every unresolved run shares its 8-byte key: jump to the first depth
        // where a member differs from the run head (or ends).
        for (uint32_t x = lane; x < size; x += 32) scratch[x] = 0xFFFFFFFFu;
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t h0 = __shfl_sync(FULL, id[0], rs[h] & 31), h1 = __shfl_sync(FULL, id[1], rs[h] & 31);
            const uint32_t hid = rs[h] < 32 ? h0 : h1;
            if (unres[h] && lane + 32 * h != rs[h]) {
                uint64_t off, offh;
                uint32_t len, lenh;
                str_of(a, id[h], off, len);
                str_of(a, hid, offh, lenh);
                uint32_t l;
                for (uint32_t d = dep[h] + 8;; d += 16) {
                    const uint64_t x0 = key8(a.chars, off, len, d), y0 = key8(a.chars, offh, lenh, d);
                    const uint64_t x1 = key8(a.chars, off, len, d + 8), y1 = key8(a.chars, offh, lenh, d + 8);
                    if (x0 != y0) { l = d + key_lcp(x0, y0); break; }
                    if (zero_byte(x0) < 8) { l = d + zero_byte(x0); break; }
                    if (x1 != y1) { l = d + 8 + key_lcp(x1, y1); break; }
                    if (zero_byte(x1) < 8) { l = d + 8 + zero_byte(x1); break; }
                }
                atomicMin(&scratch[rs[h]], l);
            }
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (unres[h]) {
                dep[h] = scratch[rs[h]];
                key[h] = key8_of(a, id[h], dep[h]);
            }
        }
        __syncwarp();
    }
}

// Segments of 2..32 strings: one warp each, four per CTA.
// dcount (graph mode): the segment count on the device; blocks stride over it.
__global__ void __launch_bounds__(128) k_warp_segs(SortState S, const Seg* segs, uint32_t nseg, const uint32_t* dcount) {
    if (dcount) nseg = *dcount;
    for (uint32_t si = blockIdx.x * 4 + (threadIdx.x >> 5); si < nseg; si += gridDim.x * 4) {
    const int lane = threadIdx.x & 31;
    const Seg seg = segs[si];
    const uint32_t* src = S.ord[seg.flags & F_PARITY];
    uint32_t id = 0;
    uint64_t key = 0;
    if ((uint32_t)lane < seg.size) {
        id = src[seg.start + lane];
        key = (seg.flags & F_KEYS) ? S.key[seg.flags & F_PARITY][seg.start + lane]
                                   : key8_of(S.a, id, seg.depth);
    }
    warp_sort(S.a, seg.size, seg.depth, key, id, S.lcp_out + seg.start);
    if ((uint32_t)lane < seg.size) S.ord_out[seg.start + lane] = id;
    }
}

template <int CAP>
constexpr size_t seg_sort_smem() {
    return (size_t)CAP * (8 + 8 + 4 + 4 + 4) + (size_t)(CAP / 2) * 3 * 4 * 2;
}

// Bucket flags inside k_seg_sort, packed above the 16-bit bucket size: the
// keys must be gathered at the bucket depth first (SF_REKEY), a pivot pass is
// due (SF_PIVOT), or the keys are pivot pseudo keys whose base depth is the
// bucket depth (SF_PSEUDO).
constexpr uint32_t SF_REKEY = 1u, SF_PIVOT = 2u, SF_PSEUDO = 4u;
constexpr uint32_t WL_MAX = 64;  // largest bucket a warp sort takes (wide splits only)

template <int CAP, int NT>
__global__ void __launch_bounds__(NT) k_seg_sort(SortState S, const Seg* segs, uint32_t nseg, const uint32_t* dcount) {
    constexpr int NW = NT / 32;
    // the 64-wide warp sort only where segments are large enough to split
    // wide (its registers would cost the small variant occupancy)
    constexpr uint32_t WIDE_WL = CAP >= 1024 ? WL_MAX : 32;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* sk = (unsigned long long*)smem;
    unsigned long long* tk = sk + CAP;
    uint32_t* so = (uint32_t*)(tk + CAP);
    uint32_t* to = so + CAP;
    uint32_t* pk = to + CAP;  // digit << 24 | rank within the warp's chunk
    uint32_t* stk = pk + CAP;  // (start, size | flags << 16, depth) of buckets > 32
    uint32_t* wl = stk + 3 * (CAP / 2);  // (start, size | flags << 16, depth) of buckets <= WL_MAX
    __shared__ uint32_t hist[256], bstart[256];
    __shared__ uint32_t wcnt[NW][256];
    __shared__ uint32_t s_top, s_nw, s_cur[3];
    __shared__ unsigned long long s_diff;
    __shared__ BitTables sbt;
    if (dcount) nseg = *dcount;
    for (uint32_t bi = blockIdx.x; bi < nseg; bi += gridDim.x) {
    const Seg seg = segs[bi];
    const uint32_t start = seg.start, size = seg.size;
    const uint32_t* src = S.ord[seg.flags & F_PARITY];
    uint32_t* lcp = S.lcp_out + start;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (seg.flags & F_KEYS) {
        const unsigned long long* ksrc = S.key[seg.flags & F_PARITY];
        for (uint32_t i = threadIdx.x; i < size; i += NT) {
            so[i] = src[start + i];
            sk[i] = ksrc[start + i];
        }
    } else {
        for (uint32_t i = threadIdx.x; i < size; i += NT) {
            const uint32_t o = src[start + i];
            so[i] = o;
            sk[i] = key8_of(S.a, o, seg.depth);
        }
    }
    if (threadIdx.x == 0) {
        s_top = 0;
        s_nw = 0;
        uint32_t* dst = size <= 32 ? wl : stk;
        dst[0] = 0;
        dst[1] = size;
        dst[2] = seg.depth;
        if (size <= 32) s_nw = 1;
        else s_top = 1;
        s_diff = 0;
    }
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) {
            if (s_top) {
                --s_top;
                s_cur[0] = stk[3 * s_top];
                s_cur[1] = stk[3 * s_top + 1];
                s_cur[2] = stk[3 * s_top + 2];
            } else {
                s_cur[1] = 0;
            }
        }
        __syncthreads();
        const uint32_t bs = s_cur[0], bn = s_cur[1] & 0xFFFFu, dep = s_cur[2];
        uint32_t fl = s_cur[1] >> 16;
        if (bn == 0) break;
        if (fl & SF_REKEY) {
            for (uint32_t i = threadIdx.x; i < bn; i += NT) sk[bs + i] = key8_of(S.a, so[bs + i], dep);
            fl = 0;
            __syncthreads();
        } else if (fl & SF_PIVOT) {
            uint64_t off0;
            uint32_t len0;
            str_of(S.a, so[bs], off0, len0);
            for (uint32_t i = threadIdx.x; i < bn; i += NT) {
                uint64_t off;
                uint32_t len;
                str_of(S.a, so[bs + i], off, len);
                sk[bs + i] = pivot_key(S.a.chars, off, len, off0, len0, dep);
            }
            fl = SF_PSEUDO;
            __syncthreads();
        }
        const bool pseudo = fl & SF_PSEUDO;
        const uint64_t k0 = sk[bs];
        uint64_t df = 0;
        for (uint32_t i = threadIdx.x; i < bn; i += NT) df |= sk[bs + i] ^ k0;
#pragma unroll
        for (int o = 16; o; o >>= 1) df |= __shfl_xor_sync(FULL, df, o);
        if (lane == 0 && df) atomicOr(&s_diff, (unsigned long long)df);
        __syncthreads();
        df = s_diff;
        if (df == 0) {
            // one key for the whole bucket: byte-identical strings (their LCP
            // is their length), or continue deeper
            uint32_t fin = 0xFFFFFFFFu, cont = 0, cfl = SF_REKEY;
            if (pseudo) {
                const uint32_t code = (uint32_t)(k0 >> 56), byte = (uint32_t)(k0 >> 48) & 0xFFu;
                if (code == PIVOT_CAP) {
                    uint64_t o0;
                    uint32_t l0;
                    str_of(S.a, so[bs], o0, l0);
                    if (l0 < dep + PIVOT_CAP) fin = l0;
                    else cont = dep + PIVOT_CAP;
                } else if (byte == 0) {
                    fin = dep + pivot_l(code);
                } else {
                    cont = dep + pivot_l(code) + 1;
                }
                cfl = SF_PIVOT;
            } else {
                const uint32_t z = zero_byte(k0);
                if (z < 8) fin = dep + z;
                else cont = dep + 8;
            }
            if (fin != 0xFFFFFFFFu) {
                for (uint32_t i = threadIdx.x + 1; i < bn; i += NT) lcp[bs + i] = fin;
            } else if (threadIdx.x == 0) {
                stk[3 * s_top] = bs;
                stk[3 * s_top + 1] = bn | (cfl << 16);
                stk[3 * s_top + 2] = cont;
                ++s_top;
            }
            __syncthreads();
            if (threadIdx.x == 0) s_diff = 0;
            __syncthreads();
            continue;
        }
        const uint32_t b = (uint32_t)(__clzll(df) >> 3);
        const uint32_t shift = 56 - 8 * b;
        // plain keys split on their top eight differing bits (seg_bits), pivot
        // pseudo keys on a byte; digit 0 holds strings that end at byte b only
        // when that byte has no constant nonzero part
        const bool bits = S.seg_bits && !pseudo;
        const BitDigit bd = bit_digit_spec(bits ? df : (0xFFull << shift));
        if (!bd.whole) bit_tables_build(sbt, bd);  // ordered by the barrier below
        const bool ended_ok = !bits || (((k0 >> shift) & 0xFFu) & ~((df >> shift) & 0xFFu)) == 0;
        for (uint32_t x = threadIdx.x; x < NW * 256; x += NT) (&wcnt[0][0])[x] = 0;
        __syncthreads();
        // stable ranks: warp w owns the contiguous chunk [w*cs, min((w+1)*cs, bn))
        const uint32_t cs = ((bn + NW - 1) / NW + 31) & ~31u;
        const uint32_t ce = min((uint32_t)(w + 1) * cs, bn);
        for (uint32_t base = (uint32_t)w * cs; base < ce; base += 32) {
            const uint32_t i = base + lane;
            const bool v = i < ce;
            const uint32_t d = v ? bit_digit(sk[bs + i], bd, sbt) : 0x100u + lane;
            const uint32_t peers = __match_any_sync(FULL, d);
            const uint32_t r = __popc(peers & ((1u << lane) - 1u));
            const uint32_t prev = v ? wcnt[w][d] : 0u;
            __syncwarp();
            if (v && lane == __ffs(peers) - 1) wcnt[w][d] = prev + __popc(peers);
            __syncwarp();
            if (v) pk[bs + i] = (d << 24) | (prev + r);
        }
        __syncthreads();
        for (uint32_t d = threadIdx.x; d < 256; d += NT) {
            uint32_t run = 0;
#pragma unroll
            for (int ww = 0; ww < NW; ++ww) {
                const uint32_t v = wcnt[ww][d];
                wcnt[ww][d] = run;
                run += v;
            }
            hist[d] = run;
        }
        __syncthreads();
        if (w == 0) {  // exclusive scan of the 256 digit totals, 8 per lane
            uint32_t v[8], sum = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                v[t] = hist[lane * 8 + t];
                sum += v[t];
            }
            uint32_t x = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, x, o);
                if (lane >= o) x += y;
            }
            uint32_t ex = x - sum;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                bstart[lane * 8 + t] = ex;
                ex += v[t];
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < bn; i += NT) {
            const uint32_t x = pk[bs + i];
            const uint32_t d = x >> 24;
            const uint32_t dest = bstart[d] + wcnt[i / cs][d] + (x & 0xFFFFFFu);
            if (dest >= bn) {  // never taken when the counts agree
                atomicExch(&S.counters[10], 1u);
                continue;
            }
            tk[bs + dest] = sk[bs + i];
            to[bs + dest] = so[bs + i];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < bn; i += NT) {
            sk[bs + i] = tk[bs + i];
            so[bs + i] = to[bs + i];
        }
        __syncthreads();
        // split by pivot code, by the byte after a pivot code's shared
        // prefix, or by a plain key byte
        const bool code_split = pseudo && b == 0;
        const uint32_t lin = pseudo ? dep + pivot_l((uint32_t)(k0 >> 56)) : dep + b;
        for (uint32_t d = threadIdx.x; d < 256; d += NT) {
            const uint32_t cnt = hist[d];
            if (!cnt) continue;
            const uint32_t c0 = bs + bstart[d];
            if (c0 != bs) {  // boundary to the previous non-empty bucket
                uint32_t l = lin;
                if (code_split || !bd.whole) {
                    uint32_t pd = d - 1;
                    while (pd > 0 && bstart[pd] == bstart[d]) --pd;
                    // pivot codes: d + min(l, l'); bit digits: the byte of the
                    // highest bit in which the two buckets' digits differ
                    l = code_split ? dep + min(pivot_l(d), pivot_l(pd))
                                   : dep + bit_digit_byte(bd, 31u - (uint32_t)__clz(d ^ pd));
                }
                lcp[c0] = l;
            }
            if (d == 0 && !code_split && ended_ok) {  // strings that end here: byte-identical
                for (uint32_t k = 1; k < cnt; ++k) lcp[c0 + k] = lin;
                continue;
            }
            if (cnt < 2) continue;
            uint32_t cd, cf;
            if (!pseudo) {
                if (S.pivot && cnt > 32 && 2 * cnt > bn) {
                    cd = dep + b + 1;  // keeps most of the bucket: pivot pass next
                    cf = SF_PIVOT;
                } else {
                    cd = dep;
                    cf = 0;
                }
            } else if (code_split) {
                if (cnt > 32) {
                    cd = dep;
                    cf = SF_PSEUDO;
                } else {
                    cd = dep + pivot_l(d);
                    if (d == PIVOT_CAP) {
                        uint64_t o0;
                        uint32_t l0;
                        str_of(S.a, so[c0], o0, l0);
                        cd = min(dep + PIVOT_CAP, l0);
                    }
                    cf = SF_REKEY;
                }
            } else {
                cd = lin + 1;
                cf = (S.pivot && cnt > 32 && 2 * cnt > bn) ? SF_PIVOT : SF_REKEY;
            }
            // Warp list: up to 32 strings, or up to WL_MAX with plain keys
            // (valid or re-gathered) from a wide split (at most 1/8 of the
            // bucket: the keys' remaining bytes are likely to tell the strings
            // apart in one network).  Narrow splits and chains stay with the
            // block: a deep 64-string bucket on one warp would work through
            // all of its runs alone, where a block pass hands them to 8 warps,
            // and a chain of long shared prefixes gets the pivot pass.
            uint32_t* dst;
            uint32_t slot;
            if (cnt <= 32 || (cnt <= WIDE_WL && 8 * cnt <= bn && !(cf & (SF_PIVOT | SF_PSEUDO)))) {
                slot = atomicAdd(&s_nw, 1u);
                dst = wl + 3 * slot;
            } else {
                slot = atomicAdd(&s_top, 1u);
                dst = stk + 3 * slot;
            }
            dst[0] = c0;
            dst[1] = cnt | (cf << 16);
            dst[2] = cd;
        }
        if (threadIdx.x == 0) s_diff = 0;
        __syncthreads();
    }
    const uint32_t nwl = s_nw;
    // buckets of up to TINY_MAX strings: one thread each
    for (uint32_t e = threadIdx.x; e < nwl; e += NT) {
        const uint32_t ws = wl[3 * e], wn = wl[3 * e + 1] & 0xFFFFu, wd = wl[3 * e + 2];
        // keys that must be gathered first stay with a warp (32 gathers at once)
        if (wn > TINY_MAX || ((wl[3 * e + 1] >> 16) & SF_REKEY)) continue;
        const bool done = wn <= 4 ? tiny_sort<4>(sk, so, lcp, ws, wn, wd) : tiny_sort<8>(sk, so, lcp, ws, wn, wd);
        if (done) wl[3 * e + 1] |= WL_DONE;
    }
    __syncthreads();
    for (uint32_t e = w; e < nwl; e += NW) {
        if (wl[3 * e + 1] & WL_DONE) continue;
        const uint32_t ws = wl[3 * e], wn = wl[3 * e + 1] & 0xFFFFu, wd = wl[3 * e + 2];
        const bool rekey = (wl[3 * e + 1] >> 16) & SF_REKEY;
        if (WIDE_WL == 32 || wn <= 32) {
            uint64_t key = 0;
            uint32_t id = 0;
            if ((uint32_t)lane < wn) {
                id = so[ws + lane];
                key = rekey ? key8_of(S.a, id, wd) : sk[ws + lane];
            }
            warp_sort(S.a, wn, wd, key, id, lcp + ws);
            if ((uint32_t)lane < wn) so[ws + lane] = id;
        } else {
            // pk of this bucket's positions is free once the block passes end
            uint64_t key[2];
            uint32_t id[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t pos = (uint32_t)lane + 32 * h;
                id[h] = 0;
                key[h] = 0;
                if (pos < wn) {
                    id[h] = so[ws + pos];
                    key[h] = rekey ? key8_of(S.a, id[h], wd) : sk[ws + pos];
                }
            }
            if constexpr (WIDE_WL > 32) warp_sort64(S.a, wn, wd, key, id, lcp + ws, pk + ws);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t pos = (uint32_t)lane + 32 * h;
                if (pos < wn) so[ws + pos] = id[h];
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < size; i += NT) S.ord_out[start + i] = so[i];
    __syncthreads();  // shared memory is reused by the next segment
    }
}

template <int CAP, int NT>
static int launch_seg_sort(const SortState& S, const Seg* segs, uint32_t n, const char* name, cudaStream_t st) {
    if (!n) return DSSS_OK;
    constexpr size_t shm = seg_sort_smem<CAP>();
    static std::atomic<uint64_t> configured{0};
    DSSS_TRY(set_smem_once(configured, k_seg_sort<CAP, NT>, (int)shm));
    DSSS_LAUNCH(name, st, k_seg_sort<CAP, NT><<<n, NT, shm, st>>>(S, segs, n, nullptr));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}


// ------------------------------------------------------- graph mode ----
// For n up to sort_graph_max_n (off by default) the MSD passes run as one CUDA graph: the pass
// is the body of a conditional WHILE node, the number of large segments and
// the parity of their list live on the device (counters[13], [12]), grids are
// the layout's capacities (blocks past the real tiles exit), and a one-thread
// kernel at the end of each pass sets the loop condition — no host round trip
// per pass.  The small-segment sorters then stride over the device counts.

// One block: per large segment its first tile and chunk (exclusive prefix
// over the list), totals into counters[8], [9]; resets the next-list count.
__global__ void __launch_bounds__(1024) k_seg_offsets(SortState S, Seg* segs, uint32_t nseg) {
    __shared__ uint32_t st_[1024], sc_[1024];
    if (!segs) {
        segs = S.large[S.counters[12]];
        nseg = S.counters[13];
    }
    const uint32_t per = (nseg + 1023) / 1024;
    const uint32_t b = min(nseg, threadIdx.x * per), e = min(nseg, b + per);
    uint32_t tt = 0, tc = 0;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t t = (segs[i].size + LT_TILE - 1) / LT_TILE;
        tt += t;
        tc += (t + CHUNK_TILES - 1) / CHUNK_TILES;
    }
    st_[threadIdx.x] = tt;
    sc_[threadIdx.x] = tc;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t vt = threadIdx.x >= (unsigned)off ? st_[threadIdx.x - off] : 0;
        const uint32_t vc = threadIdx.x >= (unsigned)off ? sc_[threadIdx.x - off] : 0;
        __syncthreads();
        st_[threadIdx.x] += vt;
        sc_[threadIdx.x] += vc;
        __syncthreads();
    }
    uint32_t rt = st_[threadIdx.x] - tt, rc = sc_[threadIdx.x] - tc;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t t = (segs[i].size + LT_TILE - 1) / LT_TILE;
        // keys folded by the previous scatter: the bits where they differ
        if (S.child && (segs[i].flags & (F_KEYS | F_PIVOT)) == F_KEYS) segs[i].diff = segs[i].kor ^ segs[i].kand;
        S.tile0[i] = rt;
        S.chunk0[i] = rc;
        rt += t;
        rc += (t + CHUNK_TILES - 1) / CHUNK_TILES;
    }
    if (threadIdx.x == 1023) {
        S.counters[8] = st_[1023];
        S.counters[9] = sc_[1023];
        if (st_[1023] > S.cap_tiles || sc_[1023] > S.cap_chunks) {
            S.counters[8] = 0;  // nothing runs; the guard stops the loop
            S.counters[9] = 0;
            S.counters[10] = 1;
        }
        S.counters[0] = 0;   // large segments of the next pass
        S.counters[11] = 0;  // of them, without keys or with a pivot pass
        S.counters[6] = 0;   // splitter tables of this pass
    }
}

__global__ void k_loop_init(SortState S, cudaGraphConditionalHandle h) {
    S.counters[12] = 0;
    S.counters[13] = S.counters[0];
    S.counters[14] = 0;
    cudaGraphSetConditional(h, S.counters[13] > 0 ? 1u : 0u);
}

// Ends a pass: the next list becomes current; loop while it is not empty,
// no guard tripped and the pass count stays sane.
__global__ void k_pass_end(SortState S, cudaGraphConditionalHandle h) {
    uint32_t next = S.counters[0];
    if (next > S.cap_large) {
        S.counters[10] = 1;
        next = 0;
    }
    S.counters[12] ^= 1u;
    S.counters[13] = next;
    const uint32_t passes = ++S.counters[14];
    if (passes > (1u << 20)) S.counters[10] = 1;
    cudaGraphSetConditional(h, (next > 0 && S.counters[10] == 0) ? 1u : 0u);
}

// Two streams per host thread and device to capture on (the caller's stream
// may be the legacy default stream, which cannot be captured); the graph is
// then launched on the caller's stream.
static int capture_streams(cudaStream_t* cap, cudaStream_t* body) {
    constexpr int MAXDEV = 64;
    thread_local cudaStream_t tl[MAXDEV][2] = {};
    int dev = 0;
    DSSS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAXDEV) return fail(DSSS_ENOTSUP, "device %d out of range", dev);
    for (int k = 0; k < 2; ++k)
        if (!tl[dev][k]) DSSS_CUDA(cudaStreamCreateWithFlags(&tl[dev][k], cudaStreamNonBlocking));
    *cap = tl[dev][0];
    *body = tl[dev][1];
    return DSSS_OK;
}

static int sort_strings_graph(const SortLayout& L, SortState S, uint64_t n, uint32_t p, const uint32_t* ids_in,
                              uint32_t* pin, cudaStream_t run_st) {
    cudaStream_t st = nullptr, bst = nullptr;
    DSSS_TRY(capture_streams(&st, &bst));
    struct Res {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        ~Res() {
            if (x) cudaGraphExecDestroy(x);
            if (g) cudaGraphDestroy(g);
        }
    } res;
    const unsigned tiles = (unsigned)L.cap_tiles, chunks = (unsigned)L.cap_chunks, large = (unsigned)L.cap_large;
    DSSS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(L.counters, 0, 16 * sizeof(uint32_t), st);
    k_init_ids<<<grid_for(n, 256), 256, 0, st>>>(S.ord[0], ids_in, n);
    k_init_segs<<<grid_for(p, 128), 128, 0, st>>>(S, L.pb, p);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
    cudaGraphConditionalHandle h{};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
    if (e == cudaSuccess) k_loop_init<<<1, 1, 0, st>>>(S, h);
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t cond = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&cond, g, deps, ndeps, &np);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &cond, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
        // the loop body: one MSD pass, captured on a second stream into the body graph
        cudaGraph_t body = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(bst, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            k_seg_offsets<<<1, 1024, 0, bst>>>(S, nullptr, 0);
            k_prefix<<<tiles, LT_NT, 0, bst>>>(S, nullptr, 0);
            k_pivot<<<tiles, LT_NT, 0, bst>>>(S, nullptr, 0);
            k_keys_diff<<<tiles, LT_NT, 0, bst>>>(S, nullptr, 0);
            if (S.split_min) k_split_sample<<<148, SPL_SAMPLE / 2, 0, bst>>>(S, nullptr, 0);
            if (S.bits) k_hist<true><<<tiles, LT_NT, 0, bst>>>(S, nullptr, 0);
            else k_hist<false><<<tiles, LT_NT, 0, bst>>>(S, nullptr, 0);
            k_chunk_sum<<<chunks, 256, 0, bst>>>(S, nullptr, 0);
            k_seg_scan<<<large, 256, 0, bst>>>(S, nullptr, 0, nullptr);
            k_scatter<<<tiles, LT_NT, SCATTER_SMEM, bst>>>(S, nullptr, 0);
            k_pass_end<<<1, 1, 0, bst>>>(S, h);
            cudaGraph_t got = nullptr;
            e = cudaStreamEndCapture(bst, &got);
        }
    }
    if (e == cudaSuccess) {
        // small segments, striding over the device counts
        k_warp_segs<<<148 * 8, 128, 0, st>>>(S, S.small[0], 0, S.counters + 1);
        k_seg_sort<256, 128><<<148 * 8, 128, seg_sort_smem<256>(), st>>>(S, S.small[1], 0, S.counters + 2);
        k_seg_sort<1024, 256><<<148 * 4, 256, seg_sort_smem<1024>(), st>>>(S, S.small[2], 0, S.counters + 3);
        k_seg_sort<4096, 256><<<148, 256, seg_sort_smem<4096>(), st>>>(S, S.small[3], 0, S.counters + 4);
        if (S.split_min) k_lcp_fix<<<148 * 4, 256, 0, st>>>(S);
        cudaMemcpyAsync(pin, L.counters, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    }
    cudaGraph_t whole = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &whole);
    res.g = whole;
    if (e != cudaSuccess || e2 != cudaSuccess)
        return fail(DSSS_EDEVICE, "string sort graph: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    DSSS_CUDA(cudaGraphInstantiate(&res.x, whole, 0));
    {
        StageTimer t("graph:sort", run_st);
        DSSS_CUDA(cudaGraphLaunch(res.x, run_st));
    }
    DSSS_CUDA(cudaStreamSynchronize(run_st));
    if (pin[10]) return fail(DSSS_EDEVICE, "string sort: internal consistency guard tripped");
    return DSSS_OK;
}

// ------------------------------------------------------------------ host ----
static Seg* large_list(const SortLayout& L, int k) { return (Seg*)L.large[k]; }
static uint32_t clamp_small_max(uint32_t m) {
    if (m == 0) m = (uint32_t)tune(TUNE_SORT_SMALL_MAX);
    return (m == 0 || m > (uint32_t)bin_cap(NBINS - 1)) ? (uint32_t)bin_cap(NBINS - 1) : (m < 2 ? 2 : m);
}

void layout_sort(Carve& c, SortLayout& L, uint64_t n, uint32_t p, uint32_t small_max) {
    small_max = clamp_small_max(small_max);
    uint64_t N = n ? n : 1;
    L.ord[0] = c.take<uint32_t>(N);
    L.ord[1] = c.take<uint32_t>(N);
    L.key[0] = c.take<unsigned long long>(N);
    L.key[1] = c.take<unsigned long long>(N);
    L.cap_large = N / (small_max + 1) + p + 1;
    L.cap_small = N / 2 + p + 1;
    L.cap_tiles = N / LT_TILE + L.cap_large + 1;
    L.cap_chunks = L.cap_tiles / CHUNK_TILES + L.cap_large + 1;
    L.large[0] = c.take<unsigned char>(L.cap_large * sizeof(Seg));
    L.large[1] = c.take<unsigned char>(L.cap_large * sizeof(Seg));
    for (int b = 0; b < NBINS; ++b) L.small[b] = c.take<unsigned char>(L.cap_small * sizeof(Seg));
    L.tile0 = c.take<uint32_t>(L.cap_large);
    L.chunk0 = c.take<uint32_t>(L.cap_large);
    L.tmp_counts = c.take<uint32_t>(2 * L.cap_large);
    L.tile_hist = c.take<uint32_t>(L.cap_tiles * 256);
    L.chunk_pre = c.take<uint32_t>(L.cap_chunks * 256);
    L.bucket = c.take<uint32_t>(L.cap_large * 257);
    // the child table: 256 slots per large segment, about 4 bytes per string
    // once large segments hold more than 256 strings (smaller cut-offs keep
    // the per-pass key reads instead)
    L.child = small_max >= 256 ? c.take<uint32_t>(L.cap_large * 256) : nullptr;
    L.counters = c.take<uint32_t>(16);
    L.pb = c.take<uint64_t>(p + 1);
    L.scan = c.take<unsigned char>(scan_scratch_bytes(L.cap_large));
    // splitter tables: segments of at least SPL_MIN_FLOOR strings per pass;
    // fix list: (position, depth) pairs (when it runs short, passes keep the
    // byte digit)
    L.cap_spl = N / SPL_MIN_FLOOR + p + 1;
    L.spl = c.take<unsigned long long>(L.cap_spl * SPL_STRIDE);
    L.cap_fix = N / 16 + 65536;
    L.fix = c.take<uint32_t>(2 * L.cap_fix);
    L.pin = nullptr;
}

int sort_strings(const SortLayout& L, const ArenaDev& a, uint64_t n, uint32_t p, const uint64_t* pb_host,
                 const uint32_t* ids_in, uint32_t* ord_out, uint32_t* lcp_out, uint32_t small_max,
                 uint32_t* pin, cudaStream_t st, unsigned long long* dig, uint32_t* dig_mask,
                 const uint32_t* seg_depth) {
    if (dig_mask) *dig_mask = 0;
    if (n == 0) return DSSS_OK;
    SortState S;
    S.a = a;
    S.ord[0] = L.ord[0];
    S.ord[1] = L.ord[1];
    S.key[0] = L.key[0];
    S.key[1] = L.key[1];
    S.ord_out = ord_out;
    S.lcp_out = lcp_out;
    Seg* large[2] = {(Seg*)L.large[0], (Seg*)L.large[1]};
    for (int b = 0; b < NBINS; ++b) S.small[b] = (Seg*)L.small[b];
    S.tile0 = L.tile0;
    S.chunk0 = L.chunk0;
    S.tmp_counts = L.tmp_counts;
    S.tile_hist = L.tile_hist;
    S.chunk_pre = L.chunk_pre;
    S.bucket = L.bucket;
    S.counters = L.counters;
    S.child = L.child;
    S.nxt = nullptr;
    S.small_max = clamp_small_max(small_max);
    S.pivot = tune(TUNE_SORT_PIVOT) ? 1u : 0u;
    S.bits = (uint32_t)tune(TUNE_SORT_BITS);
    S.seg_bits = tune(TUNE_SORT_SEG_BITS) ? 1u : 0u;
    S.first = 0;
    S.cap_large = L.cap_large;
    S.cap_small = L.cap_small;
    S.cap_tiles = L.cap_tiles;
    S.cap_chunks = L.cap_chunks;
    {
        const int64_t v = tune(TUNE_SORT_SPLIT_MIN);
        S.split_min = v <= 0 ? 0u : (uint32_t)std::min<int64_t>(std::max<int64_t>(v, SPL_MIN_FLOOR), 0xFFFFFFFFll);
    }
    S.seg_depth = seg_depth;
    S.spl = L.spl;
    S.fix = L.fix;
    S.cap_spl = L.cap_spl;
    S.cap_fix = L.cap_fix;
    S.dig = nullptr;
    S.dig_n = n;
    // the first pass reads every string when every initial segment is large
    // (none goes straight to the small sorts) and the ids are the arena's
    bool dig_all = dig && !ids_in && n <= a.n;
    for (uint32_t q = 0; dig_all && q < p; ++q)
        if (pb_host[q + 1] - pb_host[q] <= (uint64_t)clamp_small_max(small_max)) dig_all = false;

    static std::atomic<uint64_t> scatter_configured{0};
    DSSS_TRY(set_smem_once(scatter_configured, k_scatter, (int)SCATTER_SMEM));
    DSSS_CUDA(cudaMemcpyAsync(L.pb, pb_host, (p + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    if (n <= (uint64_t)tune(TUNE_SORT_GRAPH)) {
        static std::atomic<uint64_t> c256{0}, c1024{0}, c4096{0};
        DSSS_TRY(set_smem_once(c256, k_seg_sort<256, 128>, (int)seg_sort_smem<256>()));
        DSSS_TRY(set_smem_once(c1024, k_seg_sort<1024, 256>, (int)seg_sort_smem<1024>()));
        DSSS_TRY(set_smem_once(c4096, k_seg_sort<4096, 256>, (int)seg_sort_smem<4096>()));
        S.large[0] = large_list(L, 0);
        S.large[1] = large_list(L, 1);
        S.child = nullptr;  // every pass of the graph reads the keys itself
        return sort_strings_graph(L, S, n, p, ids_in, pin, st);
    }
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 16 * sizeof(uint32_t), st));
    DSSS_LAUNCH("k_init_ids", st, k_init_ids<<<grid_for(n, 256), 256, 0, st>>>(S.ord[0], ids_in, n));
    S.large[0] = large[0];
    S.large[1] = large[1];
    DSSS_LAUNCH("k_init_segs", st, k_init_segs<<<grid_for(p, 128), 128, 0, st>>>(S, L.pb, p));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    uint32_t nlarge = pin[0];
    int cur = 0;
    uint32_t guard = 0;
    S.dig = dig_all ? dig : nullptr;
    bool first_pass = true;
    S.first = 1;
    // whether the list holds a segment without keys folded by the previous
    // scatter (no keys, a pivot pass, or the first pass): only then the
    // prefix, pivot and key passes run
    bool keyless = true;
    while (nlarge) {
        if (++guard > (1u << 24)) return fail(DSSS_EDEVICE, "string sort made no progress");
        Seg* segs = large[cur];
        Seg* next = large[cur ^ 1];
        // tile / chunk indexing
        // tile / chunk indexing (and the next list's count reset): one block
        DSSS_LAUNCH("k_seg_offsets", st, k_seg_offsets<<<1, 1024, 0, st>>>(S, segs, nlarge));
        // upper bounds for the grids (kernels exit past the real counts)
        uint64_t max_tiles = std::min<uint64_t>(L.cap_tiles, n / LT_TILE + nlarge + 1);
        uint64_t max_chunks = std::min<uint64_t>(L.cap_chunks, max_tiles / CHUNK_TILES + nlarge + 1);
        S.large[0] = segs;
        S.nxt = next;
        if (keyless) {
            DSSS_LAUNCH("k_spec", st, k_spec<<<std::min<uint32_t>(nlarge, 148 * 16), 256, 0, st>>>(S, segs, nlarge));
            DSSS_LAUNCH("k_prefix", st, k_prefix<<<(unsigned)max_tiles, LT_NT, 0, st>>>(S, segs, nlarge));
            DSSS_LAUNCH("k_pivot", st, k_pivot<<<(unsigned)max_tiles, LT_NT, 0, st>>>(S, segs, nlarge));
            DSSS_LAUNCH("k_keys_diff", st, k_keys_diff<<<(unsigned)max_tiles, LT_NT, 0, st>>>(S, segs, nlarge));
        }
        if (S.split_min)
            DSSS_LAUNCH("k_split_sample", st,
                        k_split_sample<<<std::min<uint32_t>(nlarge, 148 * 2), SPL_SAMPLE / 2, 0, st>>>(S, segs, nlarge));
        // the bit-digit histogram only in passes that can split on bits (its
        // tables and registers cost the byte form's occupancy)
        if (S.bits && (S.bits != 3 || S.first))
            DSSS_LAUNCH("k_hist", st, k_hist<true><<<(unsigned)max_tiles, LT_NT, 0, st>>>(S, segs, nlarge));
        else
            DSSS_LAUNCH("k_hist", st, k_hist<false><<<(unsigned)max_tiles, LT_NT, 0, st>>>(S, segs, nlarge));
        DSSS_LAUNCH("k_chunk_sum", st, k_chunk_sum<<<(unsigned)max_chunks, 256, 0, st>>>(S, segs, nlarge));
        DSSS_LAUNCH("k_seg_scan", st, k_seg_scan<<<nlarge, 256, 0, st>>>(S, segs, nlarge, next));
        DSSS_LAUNCH("k_scatter", st, k_scatter<<<(unsigned)max_tiles, LT_NT, SCATTER_SMEM, st>>>(S, segs, nlarge));
        DSSS_CUDA(cudaGetLastError());
        DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        nlarge = pin[0];
        keyless = !S.child || pin[11] != 0;
        if (pin[10]) return fail(DSSS_EDEVICE, "string sort: internal consistency guard tripped");
        if (nlarge > L.cap_large) return fail(DSSS_EDEVICE, "string sort: large-segment list overflow");
        cur ^= 1;
        if (first_pass && S.dig && dig_mask) *dig_mask = 15u & ~pin[15];  // depths no segment skipped
        first_pass = false;
        S.first = 0;
        S.dig = nullptr;
    }
    for (int b = 0; b < NBINS; ++b)
        if (pin[1 + b] > L.cap_small) return fail(DSSS_EDEVICE, "string sort: small-segment list overflow");
    if (pin[1]) {
        DSSS_LAUNCH("k_warp_segs", st, k_warp_segs<<<(pin[1] + 3) / 4, 128, 0, st>>>(S, S.small[0], pin[1], nullptr));
        DSSS_CUDA(cudaGetLastError());
    }
    DSSS_TRY((launch_seg_sort<256, 128>(S, S.small[1], pin[2], "k_seg_sort256", st)));
    DSSS_TRY((launch_seg_sort<1024, 256>(S, S.small[2], pin[3], "k_seg_sort1024", st)));
    DSSS_TRY((launch_seg_sort<4096, 256>(S, S.small[3], pin[4], "k_seg_sort4096", st)));
    if (pin[5]) DSSS_LAUNCH("k_lcp_fix", st, k_lcp_fix<<<grid_for(std::min<uint64_t>(pin[5], L.cap_fix), 256), 256, 0, st>>>(S));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[10]) return fail(DSSS_EDEVICE, "string sort: internal consistency guard tripped");
    return DSSS_OK;
}

}  // namespace dsss
