// K7 — merge of receive containers: choose_merge / LcpStringLoserTree_
// (src/sorter/distributed/merging.hpp:66-123, src/merge/bingmann-lcp_losertree.hpp:203-480)
// on strings delivered prefix-compressed by the PD exchange (each string holds
// bytes [lcp, dp) of its DP prefix; lcp is relative to the previous string of
// the same source run, 0 at run starts).
//
//   1. string starts: from the NUL layout when the caller has no start table;
//   2. prefix decompression (the role of StringLcpContainer::extendPrefix,
//      strings/stringcontainer.hpp:248-333): bytes [0, lcp) of string o are
//      bytes of the nearest earlier string with a smaller LCP, found in
//      O(log n) on a min-tree over the LCP array, recursively;
//   3. merge rounds: runs are merged pairwise (log2 of the run count rounds)
//      with merge-path partitioning (each thread finds its diagonal split by
//      binary search, then merges 8 outputs serially); the serial merge keeps
//      the LCP of both run heads with the last output, so characters are only
//      compared when those LCPs are equal, and then only from that depth on.
// Byte-identical strings keep run order (lower source PE first).
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "merge.cuh"
#include "strsort.cuh"

namespace dsss {

constexpr uint32_t NONE32 = 0xFFFFFFFFu;
constexpr int MG_NT = 256, MG_VT = 8, MG_TILE = MG_NT * MG_VT;

__global__ void k_start_flags(const uint8_t* chars, uint64_t bytes, uint32_t* flag) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < bytes) flag[b] = (b == 0 || chars[b - 1] == 0) ? 1u : 0u;
}

__global__ void k_start_compact(const uint32_t* flag, const uint32_t* pos, uint64_t bytes, uint64_t n,
                                uint32_t* start, uint32_t* err) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bytes || !flag[b]) return;
    if (pos[b] >= n) {
        atomicExch(err, 1u);
        return;
    }
    start[pos[b]] = (uint32_t)b;
}

__global__ void k_full_len(const uint32_t* start, const uint32_t* lcp, uint64_t n, uint64_t bytes, uint32_t* flen,
                           uint32_t* err) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const uint64_t b = start[o];
    const uint64_t e = o + 1 < n ? start[o + 1] : bytes;
    if (b >= bytes || e <= b || e > bytes) {  // starts must increase inside the buffer
        atomicExch(err, 1u);
        flen[o] = lcp[o];
        return;
    }
    flen[o] = lcp[o] + (uint32_t)(e - b - 1);
}

__global__ void k_min_level(const uint32_t* prev, uint64_t nprev, uint32_t* cur, uint64_t ncur) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncur) return;
    const uint32_t a = prev[2 * i];
    const uint32_t b = 2 * i + 1 < nprev ? prev[2 * i + 1] : NONE32;
    cur[i] = min(a, b);
}

struct MinTree {
    const uint32_t* lv[40];
    uint64_t sz[40];
    int levels;
};

// Nearest j < o with lcp[j] < v, or NONE32.
__device__ uint32_t prev_smaller(const MinTree& t, uint64_t o, uint32_t v) {
    uint64_t i = o;
    for (int l = 0; l < t.levels; ++l) {
        if ((i & 1) && t.lv[l][i - 1] < v) {
            uint64_t k = i - 1;
            for (int m = l; m > 0; --m) {
                const uint64_t r = 2 * k + 1;
                k = (r < t.sz[m - 1] && t.lv[m - 1][r] < v) ? r : 2 * k;
            }
            return (uint32_t)k;
        }
        i >>= 1;
    }
    return NONE32;
}

// G lanes decompress one string together (G = 1: one thread per string), so
// that a warp's byte loads and stores fall on 32 / G strings' consecutive
// bytes instead of 32 scattered ones; strings 0, step, 2 step, ...
template <int G>
__global__ void k_extend(const uint8_t* chars, const uint32_t* start, const uint32_t* lcp, MinTree tree, uint64_t n,
                         uint64_t step, const uint64_t* foff, const uint32_t* flen, uint8_t* full, uint32_t* err) {
    const uint64_t o = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G * step;
    const uint32_t lane = threadIdx.x % G;
    if (o >= n) return;
    uint8_t* dst = full + foff[o];
    const uint32_t l0 = lcp[o];
    const uint32_t fo = flen[o];
    if (fo < l0) {
        if (lane == 0) atomicExch(err, 1u);
        return;
    }
    const uint32_t own = fo - l0;
    const uint8_t* src = chars + start[o];
#pragma unroll 4
    for (uint32_t k = lane; k < own; k += G) dst[l0 + k] = src[k];
    uint32_t need = l0;
    uint64_t cur = o;
    while (need > 0) {
        const uint32_t j = prev_smaller(tree, cur, need);
        if (j == NONE32) {  // a run must start with LCP 0
            if (lane == 0) atomicExch(err, 1u);
            return;
        }
        const uint32_t lj = lcp[j];
        if (need - lj > flen[j] - lj) {  // the LCP claims more bytes than string j holds
            if (lane == 0) atomicExch(err, 1u);
            return;
        }
        const uint8_t* sj = chars + start[j];
#pragma unroll 4
        for (uint32_t x = lj + lane; x < need; x += G) dst[x] = sj[x - lj];
        need = lj;
        cur = j;
    }
}

// A group of G lanes decompresses a chunk of XT_CHUNK consecutive strings in
// order.  The chunk's first string is decompressed beforehand (k_extend over
// every XT_CHUNK-th string, through min-tree chains, all chunks in parallel);
// every later string o copies bytes [0, lcp[o]) from string o - 1, whose first
// 32 G bytes the group keeps in shared memory (longer prefixes are read back
// from o - 1's decompressed bytes, which this group wrote before its
// __syncwarp).  Bytes [0, lcp[o]) of the buffer already hold string o - 1's
// prefix, so each string only writes its own bytes into it.  Several groups
// per warp cut the per-string overhead of short strings.
constexpr int XT_THREADS = 256, XT_CHUNK = 128;

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <int G>
__global__ void __launch_bounds__(XT_THREADS, 8)
    k_extend_chunks(const uint8_t* chars, const uint32_t* start, const uint32_t* lcp, uint64_t n, const uint64_t* foff,
                    const uint32_t* flen, uint8_t* full, uint32_t* err) {
    constexpr uint32_t GROUPS = XT_THREADS / G, BUF = 32 * G;
    __shared__ uint8_t sbuf[GROUPS][BUF];
    const uint32_t lane = threadIdx.x % G, grp = threadIdx.x / G;
    const uint32_t mask = G == 32 ? 0xffffffffu : ((1u << G) - 1) << (threadIdx.x & 31 & ~(G - 1));
    uint8_t* buf = sbuf[grp];
    const uint32_t nchunks = (uint32_t)((n + XT_CHUNK - 1) / XT_CHUNK);  // n <= bytes < 2^32
    for (uint32_t c = blockIdx.x * GROUPS + grp; c < nchunks; c += gridDim.x * GROUPS) {
        const uint32_t b0 = c * XT_CHUNK, e0 = (uint64_t)b0 + XT_CHUNK < n ? b0 + XT_CHUNK : (uint32_t)n;
        uint32_t prev_len = 0;
        const uint8_t* prev = nullptr;
        for (uint32_t g = b0; g < e0; g += G) {
            const uint32_t mine = g + lane;
            uint32_t ml = 0, mf = 0, ms = 0;
            uint64_t mo = 0;
            if (mine < e0) {
                ml = lcp[mine];
                mf = flen[mine];
                ms = start[mine];
                mo = foff[mine];
                prefetch_l1(chars + ms);
            }
            const int cnt = e0 - g < G ? (int)(e0 - g) : G;
            for (int i = 0; i < cnt; ++i) {
                const uint32_t l0 = __shfl_sync(mask, ml, i, G);
                const uint32_t fo = __shfl_sync(mask, mf, i, G);
                const uint32_t so = __shfl_sync(mask, ms, i, G);
                const uint64_t oo = __shfl_sync(mask, mo, i, G);
                uint8_t* dst = full + oo;
                if (fo < l0) {
                    if (lane == 0) atomicExch(err, 1u);
                    return;
                }
                if (g + i == b0) {  // decompressed by k_extend before this kernel
                    const uint32_t m = fo < BUF ? fo : BUF;
                    for (uint32_t x = lane; x < m; x += G) buf[x] = dst[x];
                    __syncwarp(mask);
                    prev_len = fo;
                    prev = dst;
                    continue;
                }
                if (l0 > prev_len) {  // the LCP claims more bytes than the previous string holds
                    if (lane == 0) atomicExch(err, 1u);
                    return;
                }
                for (uint32_t x = lane; x < l0; x += G) dst[x] = x < BUF ? buf[x] : prev[x];
                const uint8_t* src = chars + so;
                for (uint32_t x = l0 + lane; x < fo; x += G) {
                    const uint8_t v = src[x - l0];
                    dst[x] = v;
                    if (x < BUF) buf[x] = v;
                }
                __syncwarp(mask);
                prev_len = fo;
                prev = dst;
            }
        }
    }
}

template <int G>
static int launch_chunks(const uint8_t* chars, const uint32_t* start, const uint32_t* lcp, uint64_t n,
                         const uint64_t* foff, const uint32_t* flen, uint8_t* full, uint32_t* err, cudaStream_t st) {
    const uint64_t chunks = (n + XT_CHUNK - 1) / XT_CHUNK;
    const uint64_t groups = XT_THREADS / G;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((chunks + groups - 1) / groups, 148 * 8));
    DSSS_LAUNCH("k_extend_chunks", st,
                k_extend_chunks<G><<<grid, XT_THREADS, 0, st>>>(chars, start, lcp, n, foff, flen, full, err));
    return DSSS_OK;
}

template <int G>
static int launch_extend(const uint8_t* chars, const uint32_t* start, const uint32_t* lcp, const MinTree& tree,
                         uint64_t n, const uint64_t* foff, const uint32_t* flen, uint8_t* full, uint32_t* err,
                         cudaStream_t st, uint64_t step = 1) {
    const uint64_t strings = (n + step - 1) / step;
    DSSS_LAUNCH("k_extend", st,
                k_extend<G><<<grid_for(strings * G, 256), 256, 0, st>>>(chars, start, lcp, tree, n, step, foff, flen,
                                                                       full, err));
    return DSSS_OK;
}

// Lanes per chunk group: the knob's value, or from the average decompressed
// length (about two passes of the group over a string).
static int extend_lanes(uint64_t n, uint64_t full_bytes) {
    const int64_t k = tune(TUNE_MERGE_LANES);
    if (k > 0) return (int)k;
    const uint64_t avg = n ? full_bytes / n : 0;
    return avg <= 16 ? 4 : avg <= 48 ? 8 : avg <= 128 ? 16 : 32;
}

static int run_extend(const uint8_t* chars, const uint32_t* start, const uint32_t* lcp, const MinTree& tree,
                      uint64_t n, uint64_t full_bytes, const uint64_t* foff, const uint32_t* flen, uint8_t* full,
                      uint32_t* err, cudaStream_t st) {
    DSSS_TRY(launch_extend<4>(chars, start, lcp, tree, n, foff, flen, full, err, st, XT_CHUNK));
    switch (extend_lanes(n, full_bytes)) {
    case 4: return launch_chunks<4>(chars, start, lcp, n, foff, flen, full, err, st);
    case 8: return launch_chunks<8>(chars, start, lcp, n, foff, flen, full, err, st);
    case 16: return launch_chunks<16>(chars, start, lcp, n, foff, flen, full, err, st);
    default: return launch_chunks<32>(chars, start, lcp, n, foff, flen, full, err, st);
    }
}

// ------------------------------------------------------------------ merge ----
struct MergeJob {
    uint32_t a_beg, a_len, b_beg, b_len, out_beg, tile0;
};

struct FullView {
    const uint8_t* full;
    const uint64_t* foff;
    const uint32_t* flen;
};

// Compares strings x and y from depth h (their first h bytes are equal):
// returns <0, 0, >0 and the LCP through *l.
__device__ __forceinline__ int cmp_from(const FullView& f, uint32_t x, uint32_t y, uint32_t h, uint32_t* l) {
    const uint64_t ox = f.foff[x], oy = f.foff[y];
    const uint32_t lx = f.flen[x], ly = f.flen[y];
    for (uint32_t d = h;; d += 8) {
        const uint64_t a = key8(f.full, ox, lx, d), b = key8(f.full, oy, ly, d);
        if (a != b) {
            *l = d + key_lcp(a, b);
            return a < b ? -1 : 1;
        }
        const uint32_t z = zero_byte(a);
        if (z < 8) {
            *l = d + z;
            return 0;
        }
    }
}

__global__ void __launch_bounds__(MG_NT) k_merge_round(FullView f, const MergeJob* jobs, uint32_t njobs,
                                                       const uint32_t* ids_in, const uint32_t* lcp_in,
                                                       uint32_t* ids_out, uint32_t* lcp_out) {
    __shared__ uint32_t s_job;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = njobs;  // last job with tile0 <= blockIdx.x
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (jobs[mid].tile0 <= blockIdx.x) lo = mid;
            else hi = mid;
        }
        s_job = lo;
    }
    __syncthreads();
    const MergeJob J = jobs[s_job];
    const uint32_t total = J.a_len + J.b_len;
    const uint32_t diag = (blockIdx.x - J.tile0) * MG_TILE + threadIdx.x * MG_VT;
    if (diag >= total) return;
    const uint32_t* A = ids_in + J.a_beg;
    const uint32_t* B = ids_in + J.b_beg;
    const uint32_t* LA = lcp_in + J.a_beg;
    const uint32_t* LB = lcp_in + J.b_beg;
    // merge path: i = number of A elements among the first diag outputs (A first on ties)
    uint32_t lo = diag > J.b_len ? diag - J.b_len : 0, hi = min(diag, J.a_len);
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        uint32_t l;
        if (cmp_from(f, A[mid], B[diag - 1 - mid], 0, &l) <= 0) lo = mid + 1;
        else hi = mid;
    }
    uint32_t i = lo, j = diag - lo;
    // LCPs of both heads with the last output before this thread's range
    uint32_t ha = 0, hb = 0;
    if (diag > 0) {
        bool last_a;
        if (j == 0) last_a = true;
        else if (i == 0) last_a = false;
        else {
            uint32_t l;
            last_a = cmp_from(f, A[i - 1], B[j - 1], 0, &l) > 0;
        }
        const uint32_t last = last_a ? A[i - 1] : B[j - 1];
        uint32_t l;
        if (i < J.a_len) {
            if (last_a) ha = LA[i];
            else {
                cmp_from(f, A[i], last, 0, &l);
                ha = l;
            }
        }
        if (j < J.b_len) {
            if (!last_a) hb = LB[j];
            else {
                cmp_from(f, B[j], last, 0, &l);
                hb = l;
            }
        }
    }
    uint32_t* out_id = ids_out + J.out_beg;
    uint32_t* out_l = lcp_out + J.out_beg;
    for (uint32_t k = 0; k < MG_VT && diag + k < total; ++k) {
        bool take_a;
        uint32_t h;
        if (i >= J.a_len) {
            take_a = false;
            h = hb;
        } else if (j >= J.b_len) {
            take_a = true;
            h = ha;
        } else if (ha > hb) {
            take_a = true;
            h = ha;
        } else if (hb > ha) {
            take_a = false;
            h = hb;
        } else {
            uint32_t l;
            h = ha;
            take_a = cmp_from(f, A[i], B[j], h, &l) <= 0;
            if (take_a) hb = l;
            else ha = l;
        }
        if (take_a) {
            out_id[diag + k] = A[i];
            out_l[diag + k] = h;
            ++i;
            ha = i < J.a_len ? LA[i] : 0;
        } else {
            out_id[diag + k] = B[j];
            out_l[diag + k] = h;
            ++j;
            hb = j < J.b_len ? LB[j] : 0;
        }
    }
}

// ------------------------------------------------------------ K-way merge ----
// The p runs of each receiving PE merged at once by co-ranked tiles (knob
// merge_by_sort = 2): every KW_GAP-th string of every run is a sample; the
// samples of each receiving PE are sorted; every KW_STEP-th sorted sample B
// bounds a tile, and its rank in each run q (the number of q's strings
// before B in the merged order: bytes, then position, so that byte-identical
// strings keep run order) is found by a binary search inside the window of
// KW_GAP strings that the samples leave (the run's samples before B are
// counted from their sorted positions).  Every tile thus holds, from each
// run, the strings between two consecutive bounds: about KW_GAP * KW_STEP
// strings, at most (KW_STEP + p) * KW_GAP.  The tiles' strings are gathered
// in run order and each tile is sorted on its own from the LCP of its two
// bounds (the segment sorter, in shared memory for tiles up to 4096
// strings); the LCP at each tile's first string, with the previous tile's
// last, is computed last.
constexpr uint32_t KW_GAP = 32;
constexpr uint32_t KW_STEP = 32;

// x before y in the merged order: bytes, then position.
__device__ __forceinline__ bool kw_before(const FullView& f, uint32_t x, uint32_t y) {
    uint32_t l;
    const int c = cmp_from(f, x, y, 0, &l);
    return c < 0 || (c == 0 && x < y);
}

// Run r's samples: positions 0, KW_GAP, 2 KW_GAP, ... (one block per run).
__global__ void k_kw_samples(const uint32_t* run_begin, const uint32_t* run_len, const uint32_t* sbase, uint32_t* samp) {
    const uint32_t r = blockIdx.x;
    const uint32_t cnt = sbase[r + 1] - sbase[r];
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) samp[sbase[r] + k] = run_begin[r] + k * KW_GAP;
}

// Sorted position of every sample, stored at the sample's place (run, k).
__global__ void k_kw_posof(const uint32_t* sorted, uint64_t ns, const uint32_t* run_of, const uint32_t* run_begin,
                           const uint32_t* sbase, uint32_t* pos) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const uint32_t x = sorted[j];
    const uint32_t r = run_of[x];
    pos[sbase[r] + (x - run_begin[r]) / KW_GAP] = (uint32_t)j;
}

// One thread per (bound, run of the bound's receiving PE): the run's
// strings before the bound.  bb: first bound of each receiving PE (nrecv + 1);
// sb: first sorted sample of each receiving PE.
__global__ void k_kw_corank(FullView f, const uint32_t* sorted, const uint32_t* pos, const uint32_t* sbase,
                            const uint32_t* run_begin, const uint32_t* run_len, const uint32_t* bb, const uint64_t* sb,
                            uint32_t nrecv, uint32_t p, uint32_t* split) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nb = bb[nrecv];
    if (g >= nb * p) return;
    const uint32_t b = (uint32_t)(g / p), q = (uint32_t)(g % p);
    uint32_t lo = 0, hi = nrecv;  // receiving PE: last R with bb[R] <= b
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (bb[m] <= b) lo = m;
        else hi = m;
    }
    const uint32_t R = lo;
    const uint64_t j = sb[R] + (uint64_t)KW_STEP * (b - bb[R] + 1);  // the bound's sorted position
    const uint32_t B = sorted[j];
    const uint32_t rq = R * p + q;
    // samples of run rq sorted before the bound (their sorted positions rise)
    uint32_t a = sbase[rq], e = sbase[rq + 1];
    while (a < e) {
        const uint32_t m = (a + e) >> 1;
        if (pos[m] < j) a = m + 1;
        else e = m;
    }
    const uint32_t c = a - sbase[rq];
    uint32_t s = 0;
    if (c > 0) {
        // sample c - 1 (position (c - 1) KW_GAP) is before B, sample c (if
        // any) is not; every string between two strings shares with B at
        // least the smaller of their LCPs with B, so each comparison starts
        // there (the LCP-aware binary search)
        const uint32_t rb0 = run_begin[rq], len = run_len[rq];
        uint32_t l2 = (c - 1) * KW_GAP, h2 = min(c * KW_GAP, len);
        uint32_t llo, lhi = 0;
        cmp_from(f, rb0 + l2, B, 0, &llo);
        if (h2 < len) cmp_from(f, rb0 + h2, B, 0, &lhi);
        // without an upper string nothing bounds the LCP from below until one is found
        while (h2 - l2 > 1) {
            const uint32_t m = (l2 + h2) >> 1;
            uint32_t l;
            const int cm = cmp_from(f, rb0 + m, B, min(llo, lhi), &l);
            if (cm < 0 || (cm == 0 && rb0 + m < B)) {
                l2 = m;
                llo = l;
            } else {
                h2 = m;
                lhi = l;
            }
        }
        s = h2;
    }
    split[g] = s;
}

// One block per tile: its strings gathered in run order (the tile's range of
// every run), its first output position and its strings' shared prefix (the
// LCP of its two bounds; 0 for a receiving PE's first and last tile).
// tb: first tile of each receiving PE (nrecv + 1).
__global__ void __launch_bounds__(256) k_kw_gather(FullView f, const uint32_t* sorted, const uint32_t* split,
                                                  const uint32_t* run_begin, const uint32_t* run_len,
                                                  const uint32_t* tb, const uint32_t* bb, const uint64_t* sb,
                                                  uint32_t nrecv, uint32_t p, uint32_t* gathered, uint64_t* tstart,
                                                  uint32_t* tdepth) {
    extern __shared__ uint32_t kw_sm[];  // lo[p], pre[p + 1]
    uint32_t* lo_s = kw_sm;
    uint32_t* pre = kw_sm + p;
    const uint32_t t = blockIdx.x;
    uint32_t lo = 0, hi = nrecv;  // receiving PE: last R with tb[R] <= t
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (tb[m] <= t) lo = m;
        else hi = m;
    }
    const uint32_t R = lo, lt = t - tb[R], nbR = bb[R + 1] - bb[R];
    for (uint32_t q = threadIdx.x; q < p; q += blockDim.x) {
        const uint32_t rq = R * p + q;
        const uint32_t a = lt == 0 ? 0u : split[(uint64_t)(bb[R] + lt - 1) * p + q];
        const uint32_t e = lt == nbR ? run_len[rq] : split[(uint64_t)(bb[R] + lt) * p + q];
        lo_s[q] = a;
        pre[q + 1] = e - a;
    }
    __syncthreads();
    __shared__ unsigned long long s_first;
    if (threadIdx.x == 0) {
        pre[0] = 0;
        uint64_t first = run_begin[R * p];  // the receiving PE's first output position
        for (uint32_t q = 0; q < p; ++q) {
            first += lo_s[q];
            pre[q + 1] += pre[q];
        }
        s_first = first;
        tstart[t] = first;
        uint32_t d = 0;
        if (lt > 0 && lt < nbR) {
            uint32_t l;
            cmp_from(f, sorted[sb[R] + (uint64_t)KW_STEP * lt], sorted[sb[R] + (uint64_t)KW_STEP * (lt + 1)], 0, &l);
            d = l;
        }
        tdepth[t] = d;
    }
    __syncthreads();
    const uint64_t first = s_first;
    const uint32_t size = pre[p];
    for (uint32_t o = threadIdx.x; o < size; o += blockDim.x) {
        uint32_t a = 0, e = p;  // run: last q with pre[q] <= o
        while (e - a > 1) {
            const uint32_t m = (a + e) >> 1;
            if (pre[m] <= o) a = m;
            else e = m;
        }
        gathered[first + o] = run_begin[R * p + a] + lo_s[a] + (o - pre[a]);
    }
}

// The LCP at every tile's first string but a receiving PE's first.
__global__ void k_kw_lcp_fix(FullView f, const uint64_t* tstart, const uint32_t* tb, uint32_t nrecv,
                             const uint32_t* order, uint32_t* mlcp) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tb[nrecv]) return;
    uint32_t lo = 0, hi = nrecv;
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (tb[m] <= t) lo = m;
        else hi = m;
    }
    if (t == tb[lo]) return;  // a receiving PE's first tile: LCP 0 there
    const uint64_t at = tstart[t];
    if (at == tstart[t + 1]) return;  // an empty tile: the next one's start is the same place
    uint32_t l;
    cmp_from(f, order[at - 1], order[at], 0, &l);
    mlcp[at] = l;
}

__global__ void k_merge_init(const uint32_t* lcp, const uint8_t* run_start, uint64_t n, uint32_t* ids, uint32_t* l) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    ids[o] = (uint32_t)o;
    l[o] = run_start[o] ? 0u : lcp[o];
}

__global__ void k_merge_tags(const uint32_t* ids, const uint32_t* lcp_orig, const uint8_t* run_start,
                             const uint32_t* run_of, const uint32_t* run_begin, const uint64_t* run_offset,
                             uint32_t runs_per_recv, uint64_t n, uint32_t* old_lcp, uint32_t* perm_index,
                             uint32_t* perm_pe) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const uint32_t e = ids[o];
    if (old_lcp) old_lcp[o] = run_start[e] ? 0u : lcp_orig[e];
    const uint32_t r = run_of[e];
    if (perm_index) perm_index[o] = (uint32_t)(run_offset[r] + (e - run_begin[r]));
    if (perm_pe) perm_pe[o] = r % runs_per_recv;
}

__global__ void k_run_marks(const uint32_t* run_begin, const uint32_t* run_len, uint32_t nruns, uint8_t* run_start,
                            uint32_t* run_of) {
    const uint32_t r = blockIdx.x;
    if (r >= nruns) return;
    for (uint32_t k = threadIdx.x; k < run_len[r]; k += blockDim.x) {
        run_start[run_begin[r] + k] = k == 0 ? 1 : 0;
        run_of[run_begin[r] + k] = r;
    }
}

// Scratch of the K-way merge (sizes from the run lengths, on the host).
struct KwLayout {
    uint32_t *samp, *ssort, *slcp, *pos, *sbase, *split, *gathered, *tdepth, *bb, *tb;
    uint64_t *tstart, *sb;
    SortLayout SL;
};

struct KwPlan {
    std::vector<uint32_t> sbase, bb, tb;
    std::vector<uint64_t> sb;
    uint64_t ns = 0, nb = 0, nt = 0;
};

static KwPlan kw_plan(const std::vector<uint32_t>& rl, uint32_t nrecv, uint32_t p) {
    KwPlan P;
    const uint32_t nruns = nrecv * p;
    P.sbase.assign(nruns + 1, 0);
    for (uint32_t r = 0; r < nruns; ++r) P.sbase[r + 1] = P.sbase[r] + (rl[r] + KW_GAP - 1) / KW_GAP;
    P.sb.assign(nrecv + 1, 0);
    P.bb.assign(nrecv + 1, 0);
    P.tb.assign(nrecv + 1, 0);
    for (uint32_t R = 0; R < nrecv; ++R) {
        P.sb[R] = P.sbase[(uint64_t)R * p];
        const uint64_t ms = P.sbase[(uint64_t)(R + 1) * p] - P.sbase[(uint64_t)R * p];
        const uint32_t nbR = ms ? (uint32_t)((ms - 1) / KW_STEP) : 0u;
        P.bb[R + 1] = P.bb[R] + nbR;
        P.tb[R + 1] = P.tb[R] + nbR + 1;
    }
    P.sb[nrecv] = P.sbase[nruns];
    P.ns = P.sbase[nruns];
    P.nb = P.bb[nrecv];
    P.nt = P.tb[nrecv];
    return P;
}

static void layout_kw(Carve& c, KwLayout& K, const KwPlan& P, uint64_t n, uint32_t nrecv, uint32_t p) {
    const uint64_t ns = P.ns ? P.ns : 1;
    K.samp = c.take<uint32_t>(ns);
    K.ssort = c.take<uint32_t>(ns);
    K.slcp = c.take<uint32_t>(ns);
    K.pos = c.take<uint32_t>(ns);
    K.sbase = c.take<uint32_t>((uint64_t)nrecv * p + 1);
    K.split = c.take<uint32_t>(P.nb * p + 1);
    K.gathered = c.take<uint32_t>(n ? n : 1);
    K.tstart = c.take<uint64_t>(P.nt + 1);
    K.tdepth = c.take<uint32_t>(P.nt + 1);
    K.bb = c.take<uint32_t>(nrecv + 1);
    K.tb = c.take<uint32_t>(nrecv + 1);
    K.sb = c.take<uint64_t>(nrecv + 1);
    layout_sort(c, K.SL, n, (uint32_t)std::max<uint64_t>(P.nt, nrecv), 0);
}

static int tree_levels(uint64_t n) {
    int l = 1;
    while ((n >> (l - 1)) > 1) ++l;
    return l;
}

void layout_merge(Carve& c, MergeLayout& L, uint64_t n, uint64_t bytes, uint64_t full_bytes, uint32_t nruns) {
    const uint64_t N = n ? n : 1;
    L.start = c.take<uint32_t>(N);
    L.flag = c.take<uint32_t>(bytes ? bytes : 1);
    L.pos = c.take<uint32_t>(bytes ? bytes : 1);
    L.flen = c.take<uint32_t>(N);
    L.foff = c.take<uint64_t>(N);
    L.tree = c.take<uint32_t>(2 * N + 64);
    L.ids[0] = c.take<uint32_t>(N);
    L.ids[1] = c.take<uint32_t>(N);
    L.l[0] = c.take<uint32_t>(N);
    L.l[1] = c.take<uint32_t>(N);
    L.run_start = c.take<uint8_t>(N);
    L.run_of = c.take<uint32_t>(N);
    L.run_begin = c.take<uint32_t>(nruns + 1);
    L.run_len = c.take<uint32_t>(nruns + 1);
    L.run_offset = c.take<uint64_t>(nruns + 1);
    L.jobs = c.take<MergeJob>(nruns + 1);
    L.counters = c.take<uint32_t>(4);
    L.total64 = c.take<uint64_t>(1);
    L.scan = c.take<unsigned char>(scan_scratch_bytes(bytes > N ? bytes : N));
    // Last: the second carve (once the decompressed size is known) must not
    // move any array the first one handed out.
    L.full = c.take<uint8_t>(full_bytes + 64);
}

int lcp_merge(Ctx* ctx, const uint8_t* chars, uint64_t bytes, const uint32_t* char_start, const uint32_t* lcp,
              uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* counts, const uint64_t* offsets,
              uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp, uint32_t* perm_index, uint32_t* perm_pe,
              cudaStream_t st) {
    if (n == 0) return DSSS_OK;
    if (bytes >= (1ull << 32)) return fail(DSSS_ENOTSUP, "receive containers over 4 GiB per call");
    const uint32_t nruns = nrecv * p;
    uint64_t sum = 0;
    for (uint32_t r = 0; r < nruns; ++r) sum += counts[r];
    if (sum != n) return fail(DSSS_EINVAL, "recv_counts add up to %llu, not n = %llu", (unsigned long long)sum,
                              (unsigned long long)n);
    // sizes: decompressed bytes are known only after the lengths are summed,
    // so lay out with a first pass that reserves them last.
    Carve sz(nullptr);
    MergeLayout L;
    layout_merge(sz, L, n, bytes, 0, nruns);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c0(ctx->ws);
    layout_merge(c0, L, n, bytes, 0, nruns);
    uint32_t* pin = (uint32_t*)ctx->pin;
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 4 * sizeof(uint32_t), st));
    const uint32_t* start = char_start;
    if (!start) {
        DSSS_LAUNCH("k_start_flags", st, k_start_flags<<<grid_for(bytes, 256), 256, 0, st>>>(chars, bytes, L.flag));
        DSSS_TRY(exclusive_scan_u32(L.flag, L.pos, bytes, L.counters + 1, L.scan, st));
        DSSS_LAUNCH("k_start_compact", st,
                    k_start_compact<<<grid_for(bytes, 256), 256, 0, st>>>(L.flag, L.pos, bytes, n, L.start,
                                                                         L.counters));
        start = L.start;
    }
    // runs
    std::vector<uint32_t> rb(nruns), rl(nruns);
    std::vector<uint64_t> ro(nruns);
    {
        uint64_t b = 0;
        for (uint32_t r = 0; r < nruns; ++r) {
            rb[r] = (uint32_t)b;
            rl[r] = (uint32_t)counts[r];
            ro[r] = offsets ? offsets[r] : 0;
            b += counts[r];
        }
    }
    DSSS_CUDA(cudaMemcpyAsync(L.run_begin, rb.data(), nruns * 4, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.run_len, rl.data(), nruns * 4, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.run_offset, ro.data(), nruns * 8, cudaMemcpyHostToDevice, st));
    DSSS_LAUNCH("k_run_marks", st, k_run_marks<<<nruns, 256, 0, st>>>(L.run_begin, L.run_len, nruns, L.run_start, L.run_of));
    // LCPs with run starts forced to 0 (compute_ranges_and_set_lcp_at_start_of_range)
    DSSS_LAUNCH("k_merge_init", st, k_merge_init<<<grid_for(n, 256), 256, 0, st>>>(lcp, L.run_start, n, L.ids[0], L.l[0]));
    // decompression
    DSSS_LAUNCH("k_full_len", st, k_full_len<<<grid_for(n, 256), 256, 0, st>>>(start, L.l[0], n, bytes, L.flen, L.counters));
    DSSS_TRY(exclusive_scan_u32_to_u64(L.flen, L.foff, n, L.total64, L.scan, st));
    MinTree tree;
    tree.levels = tree_levels(n);
    if (tree.levels > 40) return fail(DSSS_ENOTSUP, "merge: too many strings");
    {
        uint64_t off = 0, m = n;
        for (int l = 0; l < tree.levels; ++l) {
            tree.lv[l] = L.tree + off;
            tree.sz[l] = m;
            off += m;
            m = (m + 1) / 2;
        }
    }
    DSSS_CUDA(cudaMemcpyAsync((void*)tree.lv[0], L.l[0], n * 4, cudaMemcpyDeviceToDevice, st));
    for (int l = 1; l < tree.levels; ++l)
        DSSS_LAUNCH("k_min_level", st,
                    k_min_level<<<grid_for(tree.sz[l], 256), 256, 0, st>>>(tree.lv[l - 1], tree.sz[l - 1],
                                                                          (uint32_t*)tree.lv[l], tree.sz[l]));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(pin + 4, L.total64, 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) return fail(DSSS_EINVAL, "merge: string starts are not increasing offsets inside the buffer, "
                                         "or the NUL layout holds more strings than n");
    if (!char_start && pin[1] != n) return fail(DSSS_EINVAL, "merge: the NUL layout holds %u strings, not n", pin[1]);
    const uint64_t full_bytes = *(const uint64_t*)(pin + 4);
    // reserve the decompressed arena behind the layout (and the string sort's
    // scratch behind it when the runs are merged by sorting)
    const int64_t mode = tune(TUNE_MERGE_SORT);  // 0 pairwise rounds, 1 one sort, 2 K-way tiles
    const bool by_sort = mode == 1;
    const bool kway = mode == 2;
    SortLayout SL;
    KwLayout K;
    KwPlan P;
    if (kway) P = kw_plan(rl, nrecv, p);
    Carve sz2(nullptr);
    layout_merge(sz2, L, n, bytes, full_bytes, nruns);
    if (by_sort) layout_sort(sz2, SL, n, nrecv, 0);
    if (kway) layout_kw(sz2, K, P, n, nrecv, p);
    if (sz2.used > ctx->ws_cap) {
        // grow: everything computed so far lives in the scratch, so recompute
        // after growing (simplest correct path; the next call reuses the size)
        DSSS_TRY(ensure_ws(ctx, sz2.used));
        return lcp_merge(ctx, chars, bytes, char_start, lcp, n, nrecv, p, counts, offsets, order, merged_lcp,
                         old_lcp, perm_index, perm_pe, st);
    }
    Carve c1(ctx->ws);
    layout_merge(c1, L, n, bytes, full_bytes, nruns);
    if (by_sort) layout_sort(c1, SL, n, nrecv, 0);
    if (kway) layout_kw(c1, K, P, n, nrecv, p);
    DSSS_TRY(run_extend(chars, start, L.l[0], tree, n, full_bytes, L.foff, L.flen, L.full, L.counters + 2, st));
    if (kway) {
        ArenaDev fa{L.full, L.foff, L.flen, n};
        const FullView f{L.full, L.foff, L.flen};
        uint32_t* mlcp = merged_lcp ? merged_lcp : L.l[1];
        DSSS_CUDA(cudaMemcpyAsync(K.sbase, P.sbase.data(), P.sbase.size() * 4, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(K.sb, P.sb.data(), P.sb.size() * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(K.bb, P.bb.data(), P.bb.size() * 4, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(K.tb, P.tb.data(), P.tb.size() * 4, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(K.tstart + P.nt, &n, 8, cudaMemcpyHostToDevice, st));
        // samples of every run, sorted per receiving PE
        DSSS_LAUNCH("k_kw_samples", st, k_kw_samples<<<nruns, 256, 0, st>>>(L.run_begin, L.run_len, K.sbase, K.samp));
        DSSS_TRY(sort_strings(K.SL, fa, P.ns, nrecv, P.sb.data(), K.samp, K.ssort, K.slcp, 0, (uint32_t*)ctx->pin, st));
        if (P.ns)
            DSSS_LAUNCH("k_kw_posof", st,
                        k_kw_posof<<<grid_for(P.ns, 256), 256, 0, st>>>(K.ssort, P.ns, L.run_of, L.run_begin, K.sbase,
                                                                       K.pos));
        // every bound's rank in every run of its receiving PE, then the tiles
        if (P.nb)
            DSSS_LAUNCH("k_kw_corank", st,
                        k_kw_corank<<<grid_for(P.nb * p, 256), 256, 0, st>>>(f, K.ssort, K.pos, K.sbase, L.run_begin,
                                                                            L.run_len, K.bb, K.sb, nrecv, p, K.split));
        DSSS_LAUNCH("k_kw_gather", st,
                    k_kw_gather<<<(unsigned)P.nt, 256, (2 * p + 1) * sizeof(uint32_t), st>>>(
                        f, K.ssort, K.split, L.run_begin, L.run_len, K.tb, K.bb, K.sb, nrecv, p, K.gathered, K.tstart,
                        K.tdepth));
        std::vector<uint64_t> ts(P.nt + 1);
        DSSS_CUDA(cudaMemcpyAsync(ts.data(), K.tstart, (P.nt + 1) * 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        // every tile sorted on its own, from its strings' shared prefix
        DSSS_TRY(sort_strings(K.SL, fa, n, (uint32_t)P.nt, ts.data(), K.gathered, order, mlcp, 0, (uint32_t*)ctx->pin,
                              st, nullptr, nullptr, K.tdepth));
        DSSS_LAUNCH("k_kw_lcp_fix", st,
                    k_kw_lcp_fix<<<grid_for(P.nt, 256), 256, 0, st>>>(f, K.tstart, K.tb, nrecv, order, mlcp));
        DSSS_LAUNCH("k_merge_tags", st,
                    k_merge_tags<<<grid_for(n, 256), 256, 0, st>>>(order, lcp, L.run_start, L.run_of, L.run_begin,
                                                                  L.run_offset, p, n, old_lcp, perm_index, perm_pe));
        pin = (uint32_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        if (pin[2]) return fail(DSSS_EINVAL, "merge: a source run does not start with LCP 0");
        return DSSS_OK;
    }
    if (by_sort) {
        // Merging sorted runs by sorting their union: each receiving PE's
        // strings are one segment of the string sort, with ids in run order so
        // that byte-identical strings keep run order (lower source PE first),
        // exactly as the merge rounds below leave them.
        std::vector<uint64_t> rbnd(nrecv + 1, n);
        for (uint32_t r = 0; r < nrecv; ++r) rbnd[r] = rb[(uint64_t)r * p];
        ArenaDev fa{L.full, L.foff, L.flen, n};
        uint32_t* mlcp = merged_lcp ? merged_lcp : L.l[1];
        DSSS_TRY(sort_strings(SL, fa, n, nrecv, rbnd.data(), nullptr, order, mlcp, 0, (uint32_t*)ctx->pin, st));
        DSSS_LAUNCH("k_merge_tags", st,
                    k_merge_tags<<<grid_for(n, 256), 256, 0, st>>>(order, lcp, L.run_start, L.run_of, L.run_begin,
                                                                  L.run_offset, p, n, old_lcp, perm_index, perm_pe));
        pin = (uint32_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        if (pin[2]) return fail(DSSS_EINVAL, "merge: a source run does not start with LCP 0");
        return DSSS_OK;
    }
    FullView f{L.full, L.foff, L.flen};
    // merge rounds: within each receiving PE, runs (2j, 2j+1) merge into one
    struct Run { uint32_t beg, len; };
    std::vector<std::vector<Run>> runs(nrecv);
    for (uint32_t r = 0; r < nrecv; ++r)
        for (uint32_t q = 0; q < p; ++q) runs[r].push_back({rb[(uint64_t)r * p + q], rl[(uint64_t)r * p + q]});
    int cur = 0;
    std::vector<MergeJob> jobs;
    for (;;) {
        bool more = false;
        for (auto& v : runs) more |= v.size() > 1;
        if (!more) break;
        jobs.clear();
        uint32_t tiles = 0;
        for (auto& v : runs) {
            std::vector<Run> next;
            for (size_t k = 0; k < v.size(); k += 2) {
                MergeJob J;
                J.a_beg = v[k].beg;
                J.a_len = v[k].len;
                J.b_beg = k + 1 < v.size() ? v[k + 1].beg : v[k].beg + v[k].len;
                J.b_len = k + 1 < v.size() ? v[k + 1].len : 0;
                J.out_beg = J.a_beg;
                J.tile0 = tiles;
                const uint32_t tot = J.a_len + J.b_len;
                if (tot) {
                    tiles += (tot + MG_TILE - 1) / MG_TILE;
                    jobs.push_back(J);
                }
                next.push_back({J.a_beg, tot});
            }
            v.swap(next);
        }
        if (!jobs.empty()) {
            DSSS_CUDA(cudaMemcpyAsync(L.jobs, jobs.data(), jobs.size() * sizeof(MergeJob), cudaMemcpyHostToDevice, st));
            DSSS_LAUNCH("k_merge_round", st,
                        k_merge_round<<<tiles, MG_NT, 0, st>>>(f, L.jobs, (uint32_t)jobs.size(), L.ids[cur], L.l[cur],
                                                              L.ids[cur ^ 1], L.l[cur ^ 1]));
            DSSS_CUDA(cudaGetLastError());
            // the job table is re-filled next round: wait for this round to read it
            DSSS_CUDA(cudaStreamSynchronize(st));
            cur ^= 1;
        }
    }
    DSSS_CUDA(cudaMemcpyAsync(order, L.ids[cur], n * 4, cudaMemcpyDeviceToDevice, st));
    if (merged_lcp) DSSS_CUDA(cudaMemcpyAsync(merged_lcp, L.l[cur], n * 4, cudaMemcpyDeviceToDevice, st));
    DSSS_LAUNCH("k_merge_tags", st,
                k_merge_tags<<<grid_for(n, 256), 256, 0, st>>>(L.ids[cur], lcp, L.run_start, L.run_of, L.run_begin,
                                                              L.run_offset, p, n, old_lcp, perm_index, perm_pe));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[2]) return fail(DSSS_EINVAL, "merge: a source run does not start with LCP 0");
    return DSSS_OK;
}

// ------------------------------------------------ whole merged strings ----
// The merge-sort path's output on the receiving side: every merged string
// whole (the decompressed arena of the merge, StringLcpContainer::extendPrefix,
// stringcontainer.hpp:248-333), NUL-terminated, back to back in merged order.

__global__ void k_merged_len1(const uint32_t* order, const uint32_t* flen, uint64_t n, uint32_t* len1) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n) len1[o] = flen[order[o]] + 1;
}

constexpr uint32_t MG_COPY_LANES = 8;
__global__ void k_merged_copy(const uint8_t* full, const uint64_t* foff, const uint32_t* flen, const uint32_t* order,
                              const uint64_t* out_off, uint64_t n, uint8_t* out, uint32_t* out_len) {
    const uint64_t o = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / MG_COPY_LANES;
    const uint32_t lane = threadIdx.x % MG_COPY_LANES;
    if (o >= n) return;
    const uint32_t id = order[o];
    const uint32_t len = flen[id];
    uint8_t* dst = out + out_off[o];
    copy_words16<MG_COPY_LANES>(dst, full + foff[id], len, lane);
    if (lane == 0) {
        dst[len] = 0;
        out_len[o] = len;
    }
}

int lcp_merge_strings(Ctx* ctx, const uint8_t* chars, uint64_t bytes, const uint32_t* char_start, const uint32_t* lcp,
                      uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* counts, const uint64_t* offsets,
                      uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp, uint32_t* perm_index,
                      uint32_t* perm_pe, uint8_t* out_chars, uint64_t out_capacity, uint64_t* out_offsets,
                      uint32_t* out_lengths, uint64_t* out_bytes, cudaStream_t st) {
    *out_bytes = 0;
    DSSS_TRY(lcp_merge(ctx, chars, bytes, char_start, lcp, n, nrecv, p, counts, offsets, order, merged_lcp, old_lcp,
                       perm_index, perm_pe, st));
    if (n == 0) return DSSS_OK;
    // the merge's arrays are where its last carve put them: the decompressed
    // arena is taken last, so a carve with its size unknown finds it too
    Carve c(ctx->ws);
    MergeLayout L;
    layout_merge(c, L, n, bytes, 0, nrecv * p);
    DSSS_LAUNCH("k_merged_len1", st, k_merged_len1<<<grid_for(n, 256), 256, 0, st>>>(order, L.flen, n, out_lengths));
    DSSS_TRY(exclusive_scan_u32_to_u64(out_lengths, out_offsets, n, L.total64, L.scan, st));
    uint64_t* pin = (uint64_t*)ctx->pin;
    DSSS_CUDA(cudaMemcpyAsync(pin, L.total64, 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    *out_bytes = pin[0];
    if (pin[0] > out_capacity)
        return fail(DSSS_EINVAL, "out_capacity %llu is below the %llu output bytes", (unsigned long long)out_capacity,
                    (unsigned long long)pin[0]);
    DSSS_LAUNCH("k_merged_copy", st,
                k_merged_copy<<<grid_for(n * MG_COPY_LANES, 256), 256, 0, st>>>(L.full, L.foff, L.flen, order,
                                                                              out_offsets, n, out_chars,
                                                                              out_lengths));
    return DSSS_OK;
}

}  // namespace dsss
