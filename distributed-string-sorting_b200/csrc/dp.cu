// K1/K2 — distinguishing-prefix rounds (computeDistinguishingPrefixes,
// src/sorter/distributed/prefix_doubling.hpp:156-198, over BloomFilter::filter,
// src/sorter/distributed/bloomfilter.hpp:1415-1556).
//
// Round at depth d over the current candidates (positions in sorted order,
// ascending), one thread per candidate (K1):
//   - length < d                       -> dp = length, retired (EOS, :1183-1186);
//   - previous position is a candidate and lcp >= d
//                                      -> dp = d, stays a candidate (LCP-local
//                                         duplicate, :1187-1197);
//   - otherwise                        -> dp = d, XXH64 of the d-byte prefix mod
//                                         2^64-1 goes into a device hash table; a
//                                         string whose successor is an LCP-local
//                                         duplicate is a root and stays (:1193-1195).
// K2 keeps every hashed candidate whose hash was inserted twice or more — the
// exact 64-bit duplicate test the reference spreads over p filter PEs with a
// range-partitioned all-to-all (:529-546, :558-656, :662-765).  Whether a
// prefix hash is shared with another candidate does not depend on which PE
// holds either string, so one table over all PEs gives the same survivors.
// Survivors are compacted in position order into the next candidate list.
#include "internal.cuh"
#include "dp.cuh"

namespace dsss {

constexpr unsigned long long EMPTY_KEY = ~0ull;  // never a filter hash (mod 2^64-1)
constexpr uint32_t NO_SLOT = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t cand_at(const uint32_t* cand, uint32_t j) { return cand ? cand[j] : j; }

__global__ void k_dp_round(ArenaDev a, const uint32_t* order, const uint32_t* lcp, const uint32_t* cand,
                           uint32_t m, uint32_t depth, uint32_t* dp, uint32_t* flag, uint32_t* slot,
                           unsigned long long* tkeys, uint8_t* tdup, uint32_t mask, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t i = cand_at(cand, j);
    const uint32_t s = order[i];
    const uint32_t L = a.len[s];
    if (depth > L) {
        dp[i] = L;
        flag[j] = 0;
        slot[j] = NO_SLOT;
        return;
    }
    dp[i] = depth;
    if (j > 0 && cand_at(cand, j - 1) == i - 1 && lcp[i] >= depth) {
        flag[j] = 1;
        slot[j] = NO_SLOT;
        return;
    }
    const bool root = j + 1 < m && cand_at(cand, j + 1) == i + 1 && lcp[i + 1] >= depth;
    const unsigned long long h = filter_hash(xxh64_dev(a.chars + a.off[s], depth));
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    // Linear probing; the table always has free slots, so a free or matching
    // slot is reached within mask + 1 probes.
    for (uint32_t probe = 0;; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            sl = NO_SLOT;
            break;
        }
        unsigned long long prev = atomicCAS(&tkeys[sl], EMPTY_KEY, h);
        if (prev == EMPTY_KEY) break;
        if (prev == h) {
            tdup[sl] = 1;
            break;
        }
        sl = (sl + 1) & mask;
    }
    flag[j] = root ? 1 : 2;
    slot[j] = sl;
}

__global__ void k_dp_query(uint32_t m, uint32_t* flag, const uint32_t* slot, const uint8_t* tdup) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    if (flag[j] == 2) flag[j] = (slot[j] != NO_SLOT && tdup[slot[j]]) ? 1 : 0;
}

__global__ void k_compact(const uint32_t* cand, uint32_t m, const uint32_t* flag, const uint32_t* pos,
                          uint32_t* next) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    if (flag[j]) next[pos[j]] = cand_at(cand, j);
}

__global__ void k_prefix_hash(ArenaDev a, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t s = ids[j];
    const uint32_t L = a.len[s];
    out[j] = filter_hash(xxh64_dev(a.chars + a.off[s], depth < L ? depth : L));
}

// Power-of-two table with at most two keys per three slots.
static uint64_t table_slots(uint64_t n) {
    uint64_t t = 1024;
    while (t < n + n / 2 + 2) t <<= 1;
    return t;
}

void layout_dp(Carve& c, DpLayout& L, uint64_t n) {
    uint64_t N = n ? n : 1;
    L.cand[0] = c.take<uint32_t>(N);
    L.cand[1] = c.take<uint32_t>(N);
    L.flag = c.take<uint32_t>(N);
    L.pos = c.take<uint32_t>(N);
    L.slot = c.take<uint32_t>(N);
    L.slots = table_slots(N);
    L.tkeys = c.take<unsigned long long>(L.slots);
    L.tdup = c.take<uint8_t>(L.slots);
    L.counters = c.take<uint32_t>(8);
    L.scan = c.take<unsigned char>(scan_scratch_bytes(N));
}

int dp_rounds(const DpLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
              uint32_t* dp, uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds, uint32_t* pin,
              cudaStream_t st) {
    uint32_t r = 0;
    if (n == 0) {
        if (rounds) *rounds = 0;
        return DSSS_OK;
    }
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 8 * sizeof(uint32_t), st));
    const uint32_t* cand = nullptr;  // round 0: every position
    uint32_t m = (uint32_t)n;
    int cur = 0;
    const uint64_t start = 8;
    uint64_t depth = start;
    for (uint64_t i = start * 2;; i *= 2) {
        if (depth > 0xFFFFFFFFull) return fail(DSSS_EINVAL, "distinguishing-prefix depth overflow");
        uint64_t slots = table_slots(m);
        DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
        DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, slots, st));
        DSSS_LAUNCH("k_dp_round", st, k_dp_round<<<grid_for(m, 256), 256, 0, st>>>(a, order, lcp, cand, m, (uint32_t)depth, dp, L.flag, L.slot,
                                                    L.tkeys, L.tdup, (uint32_t)(slots - 1), L.counters + 1));
        DSSS_LAUNCH("k_dp_query", st, k_dp_query<<<grid_for(m, 256), 256, 0, st>>>(m, L.flag, L.slot, L.tdup));
        DSSS_TRY(exclusive_scan_u32(L.flag, L.pos, m, L.counters, L.scan, st));
        DSSS_LAUNCH("k_compact", st, k_compact<<<grid_for(m, 256), 256, 0, st>>>(cand, m, L.flag, L.pos, L.cand[cur]));
        DSSS_CUDA(cudaGetLastError());
        DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        if (pin[1]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table overflow");
        m = pin[0];
        if (round_counts && r < max_rounds) round_counts[r] = m;
        ++r;
        if (m == 0) break;
        cand = L.cand[cur];
        cur ^= 1;
        depth = start + i;
    }
    if (rounds) *rounds = r;
    return DSSS_OK;
}

int prefix_hash(const ArenaDev& a, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* out,
                cudaStream_t st) {
    if (m == 0) return DSSS_OK;
    DSSS_LAUNCH("k_prefix_hash", st, k_prefix_hash<<<grid_for(m, 256), 256, 0, st>>>(a, ids, m, depth, out));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

}  // namespace dsss
