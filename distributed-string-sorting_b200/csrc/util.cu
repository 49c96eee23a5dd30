// K4 adjacent LCP and the stable multisplit used for PE / bucket projections.
#include <algorithm>

#include "internal.cuh"
#include "util.cuh"

namespace dsss {

// ---------------------------------------------------------- adjacent LCP ----
// calc_lcp of sorted neighbours (strings/stringtools.hpp:158-166).  One thread
// per pair compares 8-byte big-endian chunks; pairs still equal after
// WARP_AFTER bytes are finished by a whole warp, 32 chunks (256 bytes) per
// step with a ballot over the lanes.
constexpr uint32_t WARP_AFTER = 64;

__device__ __forceinline__ uint32_t lcp_thread(const ArenaDev& a, uint32_t s, uint32_t t, uint32_t from,
                                               uint32_t limit, bool* done) {
    uint64_t os, ot;
    uint32_t ls, lt;
    str_of(a, s, os, ls);
    str_of(a, t, ot, lt);
    for (uint32_t d = from;; d += 8) {
        if (d >= limit) { *done = false; return d; }
        uint64_t x = key8(a.chars, os, ls, d), y = key8(a.chars, ot, lt, d);
        if (x != y) { *done = true; return d + key_lcp(x, y); }
        uint32_t z = zero_byte(x);
        if (z < 8) { *done = true; return d + z; }
    }
}

__global__ void k_adjacent_lcp(ArenaDev a, const uint32_t* order, uint64_t m, uint32_t* lcp, uint32_t* longq,
                               uint32_t* nlong) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (i == 0) { lcp[0] = 0; return; }
    bool done;
    uint32_t l = lcp_thread(a, order[i - 1], order[i], 0, WARP_AFTER, &done);
    if (done) lcp[i] = l;
    else longq[atomicAdd(nlong, 1u)] = (uint32_t)i;
}

__global__ void k_adjacent_lcp_warp(ArenaDev a, const uint32_t* order, const uint32_t* longq,
                                    const uint32_t* nlong, uint32_t* lcp) {
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t total = *nlong;
    for (uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wid < total; wid += nw) {
        const uint32_t i = longq[wid];
        const uint32_t s = order[i - 1], t = order[i];
        uint64_t os, ot;
        uint32_t ls, lt;
        str_of(a, s, os, ls);
        str_of(a, t, ot, lt);
        for (uint32_t d = WARP_AFTER;; d += 256) {
            uint32_t dd = d + 8 * lane;
            uint64_t x = key8(a.chars, os, ls, dd), y = key8(a.chars, ot, lt, dd);
            uint32_t stop = x != y ? 1u : (zero_byte(x) < 8 ? 1u : 0u);
            uint32_t bal = __ballot_sync(0xffffffffu, stop);
            if (bal) {
                int first = __ffs(bal) - 1;
                if (lane == first) lcp[i] = dd + (x != y ? key_lcp(x, y) : zero_byte(x));
                break;
            }
        }
    }
}

int adjacent_lcp(const ArenaDev& a, const uint32_t* order, uint64_t m, uint32_t* lcp, uint32_t* longq,
                 uint32_t* nlong, cudaStream_t st) {
    if (m == 0) return DSSS_OK;
    DSSS_CUDA(cudaMemsetAsync(nlong, 0, sizeof(uint32_t), st));
    DSSS_LAUNCH("k_adjacent_lcp", st, k_adjacent_lcp<<<grid_for(m, 256), 256, 0, st>>>(a, order, m, lcp, longq, nlong));
    DSSS_LAUNCH("k_adjacent_lcp_warp", st, k_adjacent_lcp_warp<<<(unsigned)std::min<uint64_t>(grid_for(m * 32, 256), 148 * 16), 256, 0, st>>>(a, order, longq,
                                                                                                  nlong, lcp));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

__global__ void k_make_handles(ArenaDev a, ulonglong2* h) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n) h[i] = make_ulonglong2(a.off[i], a.len[i]);
}

void make_handles(const ArenaDev& a, ulonglong2* h, cudaStream_t st) {
    if (a.n) DSSS_LAUNCH("k_make_handles", st, k_make_handles<<<grid_for(a.n, 256), 256, 0, st>>>(a, h));
}

// ------------------------------------------------------------ multisplit ----
// Stable partition of n elements by bucket id b(i) < P: dest[i] = (elements of
// buckets < b) + (elements of bucket b before i).  Histograms are stored
// bucket-major per tile, so one flat exclusive scan yields every tile's
// starting offset per bucket.
constexpr int MS_NT = 256, MS_IPT = 8, MS_TILE = MS_NT * MS_IPT;

// Counts per warp in its own row of shared memory (P x MS_NT / 32 words):
// plain shared atomics, no match, no contention between warps.
__global__ void __launch_bounds__(MS_NT) k_ms_hist(const uint32_t* bucket, uint64_t n, uint32_t P, uint64_t tiles,
                                                  uint32_t* hist) {
    extern __shared__ uint32_t h[];
    constexpr int NW = MS_NT / 32;
    for (uint32_t b = threadIdx.x; b < P * NW; b += MS_NT) h[b] = 0;
    __syncthreads();
    const uint64_t tb = (uint64_t)blockIdx.x * MS_TILE;
    uint32_t* hw = h + (threadIdx.x >> 5) * P;
    // every bucket id of the thread loaded before the first is counted
    uint32_t dv[MS_IPT];
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        const uint64_t i = tb + (uint64_t)j * MS_NT + threadIdx.x;
        dv[j] = i < n ? bucket[i] : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j)
        if (dv[j] < P) atomicAdd(&hw[dv[j]], 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < P; b += MS_NT) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) t += h[w * P + b];
        hist[(uint64_t)b * tiles + blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(MS_NT) k_ms_scatter(const uint32_t* bucket, uint64_t n, uint32_t P, uint64_t tiles,
                                                     const uint32_t* off, uint32_t* dest) {
    extern __shared__ uint32_t sm[];
    uint32_t* base = sm;           // P
    uint32_t* wcnt = sm + P;       // (MS_NT/32) x P
    for (uint32_t b = threadIdx.x; b < P; b += MS_NT) {
        base[b] = off[(uint64_t)b * tiles + blockIdx.x];
        for (int w = 0; w < MS_NT / 32; ++w) wcnt[w * P + b] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t wb = (uint64_t)blockIdx.x * MS_TILE + (uint64_t)w * 32 * MS_IPT;
    uint32_t rk[MS_IPT];
    uint32_t bk[MS_IPT];
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        uint64_t i = wb + j * 32 + lane;
        uint32_t d = i < n ? bucket[i] : 0xFFFFFFFFu - lane;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t r = __popc(peers & ((1u << lane) - 1));
        uint32_t prev = i < n ? wcnt[w * P + d] : 0;
        __syncwarp();
        if (i < n && lane == __ffs(peers) - 1) wcnt[w * P + d] = prev + __popc(peers);
        __syncwarp();
        rk[j] = prev + r;
        bk[j] = d;
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < P; b += MS_NT) {
        uint32_t run = 0;
        for (int ww = 0; ww < MS_NT / 32; ++ww) {
            uint32_t v = wcnt[ww * P + b];
            wcnt[ww * P + b] = run;
            run += v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        uint64_t i = wb + j * 32 + lane;
        if (i < n) {
            uint32_t d = base[bk[j]] + wcnt[w * P + bk[j]] + rk[j];
            dest[i] = d < n ? d : 0xFFFFFFFFu;  // out-of-range marks a count mismatch; users check
        }
    }
}

// Same partition, carrying NPAY u32 payload columns: out_k[dest(i)] = in_k[i]
// (in_k == NULL carries i itself), rank_out[i] = position of i inside its
// bucket.  The tile is reordered by bucket in shared memory first, so global
// writes of each bucket's run are contiguous.
struct Payload {
    const uint32_t* in[3];
    uint32_t* out[3];
};

template <int NPAY>
constexpr size_t msp_smem(uint32_t P) {
    return (size_t)MS_TILE * (4 * NPAY + 2) + (size_t)P * 4 * (3 + MS_NT / 32);
}

template <int NPAY>
__global__ void __launch_bounds__(MS_NT, 5) k_ms_scatter_pay(const uint32_t* bucket, uint64_t n, uint32_t P,
                                                         uint64_t tiles, const uint32_t* off, Payload pl,
                                                         uint32_t* rank_out, uint32_t* err) {
    extern __shared__ __align__(16) uint32_t smp[];
    uint32_t* spay = smp;                                   // NPAY x MS_TILE
    uint16_t* sbk = (uint16_t*)(smp + NPAY * MS_TILE);      // MS_TILE
    uint32_t* base = (uint32_t*)(sbk + MS_TILE);            // P
    uint32_t* b0 = base + P;                                 // P
    uint32_t* tloff = b0 + P;                                // P
    uint32_t* wcnt = tloff + P;                              // (MS_NT/32) x P
    __shared__ uint32_t wsum[MS_NT / 32];
    for (uint32_t b = threadIdx.x; b < P; b += MS_NT) {
        base[b] = off[(uint64_t)b * tiles + blockIdx.x];
        b0[b] = off[(uint64_t)b * tiles];
#pragma unroll
        for (int w = 0; w < MS_NT / 32; ++w) wcnt[w * P + b] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t tb = (uint64_t)blockIdx.x * MS_TILE;
    const uint32_t tn = (uint32_t)min((uint64_t)MS_TILE, n - tb);
    const uint64_t wb = tb + (uint64_t)w * 32 * MS_IPT;
    // the payloads are loaded with the buckets, so that a tile waits for
    // DRAM once rather than once before and once after the ranking
    uint32_t rk[MS_IPT], bk[MS_IPT], pv[NPAY][MS_IPT];
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        const uint64_t i = wb + j * 32 + lane;
#pragma unroll
        for (int k = 0; k < NPAY; ++k) pv[k][j] = i < n ? (pl.in[k] ? pl.in[k][i] : (uint32_t)i) : 0u;
    }
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        const uint64_t i = wb + j * 32 + lane;
        const uint32_t d = i < n ? bucket[i] : 0xFFFFFFFFu - lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t r = __popc(peers & ((1u << lane) - 1));
        const uint32_t prev = i < n ? wcnt[w * P + d] : 0;
        __syncwarp();
        if (i < n && lane == __ffs(peers) - 1) wcnt[w * P + d] = prev + __popc(peers);
        __syncwarp();
        rk[j] = prev + r;
        bk[j] = d;
    }
    __syncthreads();
    // exclusive over warps per bucket, then over buckets within the tile
    // (each thread a contiguous run of buckets, block scan of the run sums)
    const uint32_t per = (P + MS_NT - 1) / MS_NT;
    const uint32_t c0 = min(P, threadIdx.x * per), c1 = min(P, c0 + per);
    uint32_t sum = 0;
    for (uint32_t b = c0; b < c1; ++b) {
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < MS_NT / 32; ++ww) {
            const uint32_t v = wcnt[ww * P + b];
            wcnt[ww * P + b] = run;
            run += v;
        }
        tloff[b] = run;
        sum += run;
    }
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t run = x - sum;
    for (int ww = 0; ww < w; ++ww) run += wsum[ww];
    for (uint32_t b = c0; b < c1; ++b) {
        const uint32_t v = tloff[b];
        tloff[b] = run;
        run += v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < MS_IPT; ++j) {
        const uint64_t i = wb + j * 32 + lane;
        if (i >= n) continue;
        const uint32_t d = bk[j];
        const uint32_t lp = tloff[d] + wcnt[w * P + d] + rk[j];
        if (lp >= tn) {  // never taken when the counts agree
            atomicExch(err, 1u);
            continue;
        }
#pragma unroll
        for (int k = 0; k < NPAY; ++k) spay[k * MS_TILE + lp] = pv[k][j];
        sbk[lp] = (uint16_t)d;
        if (rank_out) rank_out[i] = base[d] + wcnt[w * P + d] + rk[j] - b0[d];
    }
    __syncthreads();
    for (uint32_t xx = threadIdx.x; xx < tn; xx += MS_NT) {
        const uint32_t d = sbk[xx];
        const uint64_t dest = (uint64_t)base[d] + (xx - tloff[d]);
        if (dest >= n) {
            atomicExch(err, 1u);
            continue;
        }
#pragma unroll
        for (int k = 0; k < NPAY; ++k) pl.out[k][dest] = spay[k * MS_TILE + xx];
    }
}

static int launch_ms_hist(const uint32_t* bucket, uint64_t n, uint32_t P, uint64_t tiles, uint32_t* hist,
                          cudaStream_t st) {
    const size_t sm = (size_t)P * (MS_NT / 32) * sizeof(uint32_t);  // at most 32 KiB
    DSSS_LAUNCH("k_ms_hist", st, k_ms_hist<<<(unsigned)tiles, MS_NT, sm, st>>>(bucket, n, P, tiles, hist));
    return DSSS_OK;
}

template <int NPAY>
static int launch_ms_pay(const uint32_t* bucket, uint64_t n, uint32_t P, uint64_t tiles, const uint32_t* off,
                         const Payload& pl, uint32_t* rank_out, uint32_t* err, cudaStream_t st) {
    static std::atomic<uint64_t> configured{0};
    const size_t sm = msp_smem<NPAY>(P);
    DSSS_TRY(set_smem_once(configured, k_ms_scatter_pay<NPAY>, (int)msp_smem<NPAY>(MAX_SPLIT_BUCKETS)));
    DSSS_LAUNCH("k_ms_scatter_pay", st,
                k_ms_scatter_pay<NPAY><<<(unsigned)tiles, MS_NT, sm, st>>>(bucket, n, P, tiles, off, pl, rank_out, err));
    return DSSS_OK;
}

int multisplit_payload(const uint32_t* bucket, uint64_t n, uint32_t P, int npay, const uint32_t* const* in,
                       uint32_t* const* out, uint32_t* rank_out, uint32_t* err, void* scratch, cudaStream_t st) {
    if (n == 0) return DSSS_OK;
    if (P == 0 || P > MAX_SPLIT_BUCKETS) return fail(DSSS_ENOTSUP, "multisplit supports 1..%u buckets", MAX_SPLIT_BUCKETS);
    if (npay < 1 || npay > 3) return fail(DSSS_EINVAL, "multisplit: 1 to 3 payload columns");
    const uint64_t tiles = (n + MS_TILE - 1) / MS_TILE;
    const uint64_t cells = tiles * P;
    if (cells >= (1ull << 32)) return fail(DSSS_ENOTSUP, "multisplit: too many tiles x buckets");
    Carve c(scratch);
    uint32_t* hist = c.take<uint32_t>(cells);
    uint32_t* off = c.take<uint32_t>(cells);
    void* sc = c.take<unsigned char>(scan_scratch_bytes(cells));
    Payload pl;
    for (int k = 0; k < 3; ++k) {
        pl.in[k] = k < npay ? in[k] : nullptr;
        pl.out[k] = k < npay ? out[k] : nullptr;
    }
    DSSS_TRY(launch_ms_hist(bucket, n, P, tiles, hist, st));
    DSSS_TRY(exclusive_scan_u32(hist, off, cells, nullptr, sc, st));
    if (npay == 1) DSSS_TRY(launch_ms_pay<1>(bucket, n, P, tiles, off, pl, rank_out, err, st));
    else if (npay == 2) DSSS_TRY(launch_ms_pay<2>(bucket, n, P, tiles, off, pl, rank_out, err, st));
    else DSSS_TRY(launch_ms_pay<3>(bucket, n, P, tiles, off, pl, rank_out, err, st));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

uint64_t multisplit_scratch_bytes(uint64_t n, uint32_t P) {
    uint64_t tiles = (n + MS_TILE - 1) / MS_TILE;
    if (!tiles) tiles = 1;
    uint64_t cells = tiles * P;
    return 2 * ((cells * 4 + 255) & ~255ull) + ((scan_scratch_bytes(cells) + 255) & ~255ull) + 256;
}

int multisplit(const uint32_t* bucket, uint64_t n, uint32_t P, uint32_t* dest, void* scratch, cudaStream_t st) {
    if (n == 0) return DSSS_OK;
    if (P == 0 || P > MAX_SPLIT_BUCKETS) return fail(DSSS_ENOTSUP, "multisplit supports 1..%u buckets", MAX_SPLIT_BUCKETS);
    uint64_t tiles = (n + MS_TILE - 1) / MS_TILE;
    uint64_t cells = tiles * P;
    if (cells >= (1ull << 32)) return fail(DSSS_ENOTSUP, "multisplit: too many tiles x buckets");
    Carve c(scratch);
    uint32_t* hist = c.take<uint32_t>(cells);
    uint32_t* off = c.take<uint32_t>(cells);
    void* sc = c.take<unsigned char>(scan_scratch_bytes(cells));
    const size_t sh2 = (size_t)P * (1 + MS_NT / 32) * sizeof(uint32_t);
    static std::atomic<uint64_t> configured{0};
    DSSS_TRY(set_smem_once(configured, k_ms_scatter, (int)(MAX_SPLIT_BUCKETS * (1 + MS_NT / 32) * sizeof(uint32_t))));
    DSSS_TRY(launch_ms_hist(bucket, n, P, tiles, hist, st));
    DSSS_TRY(exclusive_scan_u32(hist, off, cells, nullptr, sc, st));
    DSSS_LAUNCH("k_ms_scatter", st, k_ms_scatter<<<(unsigned)tiles, MS_NT, sh2, st>>>(bucket, n, P, tiles, off, dest));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

}  // namespace dsss
