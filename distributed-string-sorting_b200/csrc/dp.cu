// K1/K2 — distinguishing-prefix rounds (computeDistinguishingPrefixes,
// src/sorter/distributed/prefix_doubling.hpp:156-198, over BloomFilter::filter,
// src/sorter/distributed/bloomfilter.hpp:1415-1556).
//
// Round at depth d, one thread per sorted position, candidates marked in a
// state byte array (K1):
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
// The hash table is sized by the number of strings hashed in the round.
#include "internal.cuh"
#include "dp.cuh"
#include "util.cuh"
#include <algorithm>

namespace dsss {

constexpr unsigned long long EMPTY_KEY = ~0ull;  // never a filter hash (mod 2^64-1)
constexpr uint32_t NO_SLOT = 0xFFFFFFFFu;
constexpr unsigned FULLM = 0xffffffffu;

// Candidate state per sorted position: st[i] = 1 while string i is a candidate.
// kind[i] after classification: 0 retired or not a candidate, 1 LCP-local
// duplicate (stays), 2 hashed (stays iff its hash is shared), 3 hashed root
// (stays; its hash is still inserted so others can collide with it).

// Length and char offset of every sorted position, gathered once per call so
// that the hash rounds read them in order.
// Four independent gathers in flight per thread (positions i, i + T, i + 2T,
// i + 3T for T threads in the grid).
constexpr int LENS_ILP = 4;
__global__ void k_dp_lens(ArenaDev a, const uint32_t* order, uint64_t n, uint32_t* lens, uint64_t* soff) {
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s[LENS_ILP];
#pragma unroll
    for (int q = 0; q < LENS_ILP; ++q) {
        const uint64_t i = i0 + q * T;
        s[q] = i < n ? order[i] : 0u;
    }
    uint64_t off[LENS_ILP];
    uint32_t len[LENS_ILP];
#pragma unroll
    for (int q = 0; q < LENS_ILP; ++q) {
        const uint64_t i = i0 + q * T;
        off[q] = 0;
        len[q] = 0;
        if (i < n) str_of(a, s[q], off[q], len[q]);
    }
#pragma unroll
    for (int q = 0; q < LENS_ILP; ++q) {
        const uint64_t i = i0 + q * T;
        if (i < n) {
            lens[i] = len[q];
            soff[i] = off[q];
        }
    }
}

static unsigned lens_grid(uint64_t n) { return grid_for((n + LENS_ILP - 1) / LENS_ILP, 256); }

// The shortest string of the arena into *out (set to ~0 beforehand): rounds
// at depths up to it retire no string at its end, so they need no lengths in
// sorted order.
__global__ void __launch_bounds__(256) k_min_len(const uint32_t* len, const ulonglong2* h, uint64_t n,
                                                 uint32_t* out) {
    uint32_t m = 0xFFFFFFFFu;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (len) {  // the 4-byte lengths, four loads in flight per thread
        for (uint64_t i = i0; i < n; i += 4 * stride) {
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] = i + q * stride < n ? len[i + q * stride] : 0xFFFFFFFFu;
#pragma unroll
            for (int q = 0; q < 4; ++q) m = min(m, v[q]);
        }
    } else {
        for (uint64_t i = i0; i < n; i += stride) m = min(m, (uint32_t)h[i].y);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m != 0xFFFFFFFFu) atomicMin(out, m);
}

// The smallest over sorted positions of max(lcp[i], lcp[i + 1]) (lcp[0] and
// lcp[n] taken as 0)
// into *out (set to ~0 beforehand): while every string is a candidate, a
// round at a depth up to it and up to the shortest string finds every string
// an LCP-local duplicate or a root, so all stay and nothing it hashes can
// matter (no string's survival rests on a hash).
__global__ void __launch_bounds__(256) k_min_nbr_lcp(const uint32_t* lcp, uint64_t n, uint32_t* out) {
    uint32_t m = 0xFFFFFFFFu;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        m = min(m, max(i ? lcp[i] : 0u, i + 1 < n ? lcp[i + 1] : 0u));  // position 0 has no predecessor
#pragma unroll
    for (int o = 16; o; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m != 0xFFFFFFFFu) atomicMin(out, m);
}

// Index of the string set holding sorted position i (set_begin: nsets+1 bounds).
__device__ __forceinline__ uint32_t set_of(const uint64_t* set_begin, uint32_t nsets, uint64_t i) {
    uint32_t lo = 0, hi = nsets;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (set_begin[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Adds the block's number of true flags to *ctr with one atomic per block
// (blockDim.x == 256, called by every thread of the block).
__device__ __forceinline__ void block_count(uint32_t* ctr, bool flag) {
    __shared__ uint32_t part[8];
    const uint32_t b = __ballot_sync(FULLM, flag);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += part[w];
        if (t) atomicAdd(ctr, t);
    }
    __syncthreads();
}

// Grid of the grid-stride kernels: up to eight 256-thread blocks per SM.
static unsigned stride_grid(uint64_t n) { return (unsigned)std::min<uint64_t>(grid_for(n, 256), 148 * 8); }

// Adds v (per thread) over the block to *ctr with one atomic per block
// (blockDim.x == 256, called by every thread of the block).
__device__ __forceinline__ void block_add(uint32_t* ctr, uint32_t v) {
    __shared__ uint32_t part[8];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULLM, v, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += part[w];
        if (t) atomicAdd(ctr, t);
    }
    __syncthreads();
}

// Sets string s's bit in an arena-order bitmap (the strings hashed by a
// dense round, which runs in arena order).
__device__ __forceinline__ void mark_string(uint32_t* m, uint32_t s) { atomicOr(&m[s >> 5], 1u << (s & 31)); }

// Marks every hashed string of a dense round (kinds 2 and 3) in the
// arena-order bitmap, when not every string of the arena is hashed.
__global__ void __launch_bounds__(256) k_dp_mark(const uint8_t* kind, const uint32_t* order, uint64_t n,
                                                 uint32_t* hmask) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && kind[i] >= 2) mark_string(hmask, order[i]);
}

// Grid-stride over positions (grid a few blocks per SM): one pair of counter
// atomics per block instead of per 256 positions.  hmask (with order): every
// hashed string is marked for the arena-order form of the round (an atomic
// OR into a bitmap of n bits, which stays in L2; random byte stores into a
// byte per string measured slower).  lens (the
// lengths in sorted order) may be null when every string reaches depth.
__global__ void __launch_bounds__(256) k_dp_classify(const uint8_t* st, int all, const uint32_t* lens,
                                                     const uint32_t* lcp, uint64_t n, uint32_t depth, uint32_t* dp,
                                                     uint8_t* st_next, uint8_t* kind, uint32_t* counters,
                                                     const uint64_t* set_begin, uint32_t nsets, uint32_t* set_cnt,
                                                     const uint32_t* order = nullptr, uint32_t* hmask = nullptr) {
    uint32_t nhashed = 0, nstays = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x % 32 < n; i += stride) {
        bool hashed = false;
        if (i < n) {
            uint8_t k = 0, nx = 0;
            if (all || st[i]) {
                const uint32_t L = lens ? lens[i] : 0xFFFFFFFFu;  // no lengths: none ends before depth
                if (depth > L) {
                    dp[i] = L;  // end of string before the depth (EOS)
                } else {
                    dp[i] = depth;
                    if (i > 0 && (all || st[i - 1]) && lcp[i] >= depth) {
                        k = 1;
                        nx = 1;
                    } else {
                        const bool root = i + 1 < n && (all || st[i + 1]) && lcp[i + 1] >= depth;
                        k = root ? 3 : 2;
                        nx = root ? 1 : 0;
                        hashed = true;
                    }
                }
            }
            kind[i] = k;
            st_next[i] = nx;
            nstays += nx;
            nhashed += hashed;
            if (hashed && hmask) mark_string(hmask, order[i]);
        }
        if (nsets > 1) {  // hashed strings per set size the per-set table regions
            const int lane = threadIdx.x & 31;
            const uint32_t sid = hashed ? set_of(set_begin, nsets, i) : 0xFFFFFFFFu - lane;
            const uint32_t peers = __match_any_sync(FULLM, sid);
            if (hashed && lane == __ffs(peers) - 1) atomicAdd(&set_cnt[sid], (uint32_t)__popc(peers));
        }
    }
    block_add(counters + 0, nhashed);
    block_add(counters + 1, nstays);
}

// k_dp_classify for one string set over 16-byte-aligned arrays: four
// consecutive positions per thread, read and written as vectors (the same
// per-position rule; st of the neighbours i - 1 and i + 4 read singly).
__global__ void __launch_bounds__(256) k_dp_classify4(const uint8_t* st, int all, const uint32_t* lens,
                                                      const uint32_t* lcp, uint64_t n, uint32_t depth, uint32_t* dp,
                                                      uint8_t* st_next, uint8_t* kind, uint32_t* counters,
                                                      const uint32_t* order = nullptr, uint32_t* hmask = nullptr) {
    uint32_t nhashed = 0, nstays = 0;
    const uint64_t groups = n >> 2;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < groups; t += stride) {
        const uint64_t i0 = t * 4;
        const uint4 L4 = lens ? reinterpret_cast<const uint4*>(lens)[t] : make_uint4(~0u, ~0u, ~0u, ~0u);
        const uint4 C4 = reinterpret_cast<const uint4*>(lcp)[t];
        const uint32_t Ls[4] = {L4.x, L4.y, L4.z, L4.w};
        const uint32_t Cs[5] = {C4.x, C4.y, C4.z, C4.w, i0 + 4 < n ? lcp[i0 + 4] : 0u};
        uint8_t S[6];  // st[i0 - 1 .. i0 + 4]
        if (all) {
#pragma unroll
            for (int q = 0; q < 6; ++q) S[q] = 1;
        } else {
            const uchar4 s4 = reinterpret_cast<const uchar4*>(st)[t];
            S[0] = i0 > 0 ? st[i0 - 1] : 0;
            S[1] = s4.x;
            S[2] = s4.y;
            S[3] = s4.z;
            S[4] = s4.w;
            S[5] = i0 + 4 < n ? st[i0 + 4] : 0;
        }
        uint32_t D[4];
        uint8_t K[4], X[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint64_t i = i0 + q;
            uint8_t k = 0, nx = 0;
            D[q] = 0xFFFFFFFFu;  // untouched
            if (S[q + 1]) {
                const uint32_t L = Ls[q];
                if (depth > L) {
                    D[q] = L;
                } else {
                    D[q] = depth;
                    if (i > 0 && S[q] && Cs[q] >= depth) {
                        k = 1;
                        nx = 1;
                    } else {
                        const bool root = i + 1 < n && S[q + 2] && Cs[q + 1] >= depth;
                        k = root ? 3 : 2;
                        nx = root ? 1 : 0;
                        ++nhashed;
                    }
                }
            }
            K[q] = k;
            X[q] = nx;
            nstays += nx;
            if (k >= 2 && hmask) mark_string(hmask, order[i]);
        }
        if (all) {
            reinterpret_cast<uint4*>(dp)[t] = make_uint4(D[0], D[1], D[2], D[3]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (D[q] != 0xFFFFFFFFu) dp[i0 + q] = D[q];
        }
        reinterpret_cast<uchar4*>(kind)[t] = make_uchar4(K[0], K[1], K[2], K[3]);
        reinterpret_cast<uchar4*>(st_next)[t] = make_uchar4(X[0], X[1], X[2], X[3]);
    }
    // the last n % 4 positions, one thread each
    const uint64_t tail = groups * 4;
    const uint64_t tt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tt < n - tail) {
        const uint64_t i = tail + tt;
        uint8_t k = 0, nx = 0;
        if (all || st[i]) {
            const uint32_t L = lens ? lens[i] : 0xFFFFFFFFu;
            if (depth > L) {
                dp[i] = L;
            } else {
                dp[i] = depth;
                if (i > 0 && (all || st[i - 1]) && lcp[i] >= depth) {
                    k = 1;
                    nx = 1;
                } else {
                    const bool root = i + 1 < n && (all || st[i + 1]) && lcp[i + 1] >= depth;
                    k = root ? 3 : 2;
                    nx = root ? 1 : 0;
                    ++nhashed;
                    if (hmask) mark_string(hmask, order[i]);
                }
            }
        }
        kind[i] = k;
        st_next[i] = nx;
        nstays += nx;
    }
    block_add(counters + 0, nhashed);
    block_add(counters + 1, nstays);
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// Inserts h into the table region (base, mask) by linear probing; returns its
// slot, NO_SLOT when the region is full.  The table always has free slots, so
// a free or matching slot is reached within mask + 1 probes.
__device__ __forceinline__ uint32_t table_insert(unsigned long long* tkeys, uint8_t* tdup, uint64_t base, uint32_t mask,
                                                 unsigned long long h, uint32_t* err, uint32_t* ndup) {
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    for (uint32_t probe = 0;; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            return NO_SLOT;
        }
        const unsigned long long prev = atomicCAS(&tkeys[base + sl], EMPTY_KEY, h);
        if (prev == EMPTY_KEY) break;
        if (prev == h) {
            tdup[base + sl] = 1;
            atomicAdd(ndup, 1u);
            break;
        }
        sl = (sl + 1) & mask;
    }
    return (uint32_t)(base + sl);
}

// Each string set owns a power-of-two region of the table (base, mask): equal
// prefixes in different sets are not duplicates of each other.
__global__ void __launch_bounds__(256, 5) k_dp_hash(ArenaDev a, const uint64_t* soff, const uint8_t* kind, uint64_t n, uint32_t depth,
                          unsigned long long* tkeys, uint8_t* tdup, uint32_t mask1, const uint64_t* set_begin,
                          uint32_t nsets, const uint64_t* set_base, const uint32_t* set_mask, uint32_t* slot,
                          uint32_t* err, uint32_t* ndup) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] < 2) return;
    uint64_t base = 0;
    uint32_t mask = mask1;
    if (nsets > 1) {
        const uint32_t sid = set_of(set_begin, nsets, i);
        base = set_base[sid];
        mask = set_mask[sid];
    }
    const unsigned long long h = filter_hash(xxh64_dev(a.chars + soff[i], depth));
    slot[i] = table_insert(tkeys, tdup, base, mask, h, err, ndup);
}

// k_dp_hash for rounds that hash few positions (e.g. only the roots of long
// runs of LCP-local duplicates): a few blocks per SM stride over the kind
// array, 16 positions per 16-byte load, instead of one thread per position.
// Without the gathered offsets (soff null) each hashed position finds its
// string through order.
__global__ void __launch_bounds__(256) k_dp_hash_sparse(ArenaDev a, const uint64_t* soff, const uint32_t* order,
                                                        const uint8_t* kind, uint64_t n,
                                                        uint32_t depth, unsigned long long* tkeys, uint8_t* tdup,
                                                        uint32_t mask1, const uint64_t* set_begin, uint32_t nsets,
                                                        const uint64_t* set_base, const uint32_t* set_mask,
                                                        uint32_t* slot, uint32_t* err, uint32_t* ndup) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t groups = (n + 15) / 16;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += stride) {
        uint32_t w[4];
        if (g * 16 + 16 <= n) {  // kind is 16-byte aligned (scratch carving)
            const uint4 v = reinterpret_cast<const uint4*>(kind)[g];
            w[0] = v.x;
            w[1] = v.y;
            w[2] = v.z;
            w[3] = v.w;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                w[q] = 0;
                for (int b = 0; b < 4; ++b) {
                    const uint64_t i = g * 16 + 4 * q + b;
                    if (i < n) w[q] |= (uint32_t)kind[i] << (8 * b);
                }
            }
        }
        // kinds are 0..3: bit 1 of a byte marks a hashed position
        if (!((w[0] | w[1] | w[2] | w[3]) & 0x02020202u)) continue;
        for (int b = 0; b < 16; ++b) {
            if (!((w[b >> 2] >> (8 * (b & 3))) & 2u)) continue;
            const uint64_t i = g * 16 + b;
            uint64_t base = 0;
            uint32_t mask = mask1;
            if (nsets > 1) {
                const uint32_t sid = set_of(set_begin, nsets, i);
                base = set_base[sid];
                mask = set_mask[sid];
            }
            uint64_t off;
            if (soff) {
                off = soff[i];
            } else {
                uint32_t len;
                str_of(a, order[i], off, len);
            }
            const unsigned long long h = filter_hash(xxh64_dev(a.chars + off, depth));
            slot[i] = table_insert(tkeys, tdup, base, mask, h, err, ndup);
        }
    }
}

// One hash round's launch: the sparse form when fewer than 1/8 of the
// positions hash (soff may then be null: offsets through order), else the
// dense form (soff required).
static bool sparse_round(uint64_t hashed, uint64_t n) { return hashed * 8 < n; }

static int launch_dp_hash(const ArenaDev& a, const uint64_t* soff, const uint32_t* order, const uint8_t* kind,
                          uint64_t n, uint32_t depth,
                          uint64_t hashed, unsigned long long* tkeys, uint8_t* tdup, uint32_t mask1,
                          const uint64_t* set_begin, uint32_t nsets, const uint64_t* set_base,
                          const uint32_t* set_mask, uint32_t* slot, uint32_t* err, uint32_t* ndup,
                          cudaStream_t st) {
    if (sparse_round(hashed, n)) {
        DSSS_LAUNCH("k_dp_hash", st,
                    k_dp_hash_sparse<<<stride_grid((n + 15) / 16), 256, 0, st>>>(a, soff, order, kind, n, depth, tkeys,
                                                                     tdup, mask1,
                                                                     set_begin, nsets, set_base, set_mask, slot, err,
                                                                     ndup));
    } else {
        DSSS_LAUNCH("k_dp_hash", st,
                    k_dp_hash<<<grid_for(n, 256), 256, 0, st>>>(a, soff, kind, n, depth, tkeys, tdup, mask1, set_begin,
                                                               nsets, set_base, set_mask, slot, err, ndup));
    }
    return DSSS_OK;
}

// Split form of k_dp_hash (knob dp_split): the hashes first, stored per
// position, then the table inserts by a kernel of few registers, so that many
// more inserts are in flight.
__global__ void __launch_bounds__(256, 5) k_dp_hash_store(ArenaDev a, const uint64_t* soff, const uint8_t* kind,
                                                          uint64_t n, uint32_t depth, unsigned long long* hbuf) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] < 2) return;
    hbuf[i] = filter_hash(xxh64_dev(a.chars + soff[i], depth));
}

__global__ void __launch_bounds__(256) k_dp_insert(const uint8_t* kind, uint64_t n, const unsigned long long* hbuf,
                                                   unsigned long long* tkeys, uint8_t* tdup, uint32_t mask1,
                                                   const uint64_t* set_begin, uint32_t nsets, const uint64_t* set_base,
                                                   const uint32_t* set_mask, uint32_t* slot, uint32_t* err,
                                                   uint32_t* ndup) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] < 2) return;
    uint64_t base = 0;
    uint32_t mask = mask1;
    if (nsets > 1) {
        const uint32_t sid = set_of(set_begin, nsets, i);
        base = set_base[sid];
        mask = set_mask[sid];
    }
    slot[i] = table_insert(tkeys, tdup, base, mask, hbuf[i], err, ndup);
}

// Dense hash rounds (at least 1/dp_digest of the positions hash) run in arena
// order.  The classification marks every hashed string (kinds 2 and 3) in the
// arena-order bitmap hmask; k_dp_arena_insert walks the strings front to
// back, so the d-byte prefixes are read in address order (at the first
// schedule depths it reads the hashes the string sort's first pass stored
// instead), and inserts the hash of every marked string into the table.  The first insert of a hash
// owns its slot (tid); an equal later insert marks the slot shared and its
// own string in the arena-order bitmap dmask.  k_dp_owner_dups then adds the
// owners of shared slots to dmask, and k_dp_query_mask keeps every kind-2
// position whose string is in dmask.  The table receives the same hashes as
// in the sorted-order form, so every string gets the same outcome; no
// per-string state is gathered by sorted position except the one bit read
// back by the query.
__device__ __forceinline__ bool bit_of(const uint32_t* m, uint64_t s) { return (m[s >> 5] >> (s & 31)) & 1u; }

__global__ void __launch_bounds__(256) k_dp_arena_insert(ArenaDev a, uint32_t depth, const unsigned long long* dig,
                                                         const uint32_t* hmask,
                                                         unsigned long long* tkeys, uint8_t* tdup, uint32_t* tid,
                                                         uint32_t mask1, const uint64_t* set_begin, uint32_t nsets,
                                                         const uint64_t* set_base, const uint32_t* set_mask,
                                                         uint32_t* dmask, uint32_t* err, uint32_t* ndup,
                                                         uint32_t check, uint32_t* bad) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n || (hmask && !bit_of(hmask, s))) return;
    unsigned long long h;
    if (dig) {  // stored by the string sort's first pass
        h = dig[s];
        if (check) {
            uint64_t off;
            uint32_t L;
            str_of(a, (uint32_t)s, off, L);
            if (h != filter_hash(xxh64_dev(a.chars + off, depth))) atomicExch(bad, 1u);
        }
    } else {
        uint64_t off;
        uint32_t L;
        str_of(a, (uint32_t)s, off, L);
        h = filter_hash(xxh64_dev(a.chars + off, depth));
    }
    uint64_t base = 0;
    uint32_t mask = mask1;
    if (nsets > 1) {  // a set's strings occupy the same index range in the arena and in the order
        const uint32_t sid = set_of(set_begin, nsets, s);
        base = set_base[sid];
        mask = set_mask[sid];
    }
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    for (uint32_t probe = 0;; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            return;
        }
        const unsigned long long prev = atomicCAS(&tkeys[base + sl], EMPTY_KEY, h);
        if (prev == EMPTY_KEY) {
            tid[base + sl] = (uint32_t)s;
            return;
        }
        if (prev == h) {
            tdup[base + sl] = 1;
            atomicAdd(ndup, 1u);
            atomicOr(&dmask[s >> 5], 1u << (s & 31));
            return;
        }
        sl = (sl + 1) & mask;
    }
}

// Dense rounds without a hash table in DRAM (whose random atomics bound the
// round): the hashed strings' (hash, string) pairs are partitioned in arena
// order into 2^B buckets by the hash's top B bits, PD_TARGET pairs per bucket
// on average, by two radix passes (top b1 <= 8 bits, then the next b2 = B - b1
// bits inside each coarse bucket): per tile a shared-memory histogram, one
// exclusive scan over the bucket-major (bucket, tile) counts, and a scatter
// to each (bucket, tile)'s range with shared-memory cursors — no global
// atomic per pair.  One block per bucket then finds the equal hashes of its
// bucket in shared memory (68 KiB: three blocks per SM).  A bucket of more
// than PD_CAP pairs (the mean plus 45 standard deviations for uniform
// hashes; only many equal prefixes on different PEs can reach it) sends the
// round to the table form.
constexpr uint32_t PD_TARGET = 2048;
constexpr uint32_t PD_CAP = 4096;
constexpr uint32_t PD_TAB = 2 * PD_CAP;  // shared-memory slots per bucket (load <= 1/2)
constexpr uint32_t PD_NT = 512;
constexpr size_t PD_SMEM = (size_t)PD_CAP * 8 + (size_t)PD_TAB * 4 + PD_CAP;
constexpr int PP_NT = 256, PP_IPT = 16, PP_TILE = PP_NT * PP_IPT;  // positions or pairs per tile

static uint32_t pd_buckets(uint64_t hashed) {
    uint32_t nb = 1;
    while ((uint64_t)nb * PD_TARGET < hashed) nb <<= 1;
    return nb;
}

// The round's hashes of the hashed strings, in arena order, when the string
// sort's first pass did not store them (or, check, to compare with them).
__global__ void __launch_bounds__(256) k_dp_arena_hash(ArenaDev a, uint32_t depth, const unsigned long long* dig,
                                                       const uint32_t* hmask, unsigned long long* out, uint32_t* bad) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n || (hmask && !bit_of(hmask, s))) return;
    uint64_t off;
    uint32_t L;
    str_of(a, (uint32_t)s, off, L);
    const unsigned long long h = filter_hash(xxh64_dev(a.chars + off, depth));
    if (dig && h != dig[s]) atomicExch(bad, 1u);
    out[s] = h;
}

// Pass 1 counts: per tile of PP_TILE arena positions, the hashed strings per
// coarse bucket (top b1 bits), stored bucket-major: hist[b * ntiles + tile].
__global__ void __launch_bounds__(PP_NT) k_pp_hist1(uint64_t n, const unsigned long long* dig, const uint32_t* hmask,
                                                   uint32_t b1, uint32_t ntiles, uint32_t* hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * PP_TILE;
    // the mask words and the hashes loaded together (every position has a
    // hash slot; only marked ones count)
#pragma unroll 4
    for (int j = 0; j < PP_IPT; ++j) {
        const uint64_t s = t0 + (uint64_t)j * PP_NT + threadIdx.x;
        if (s < n) {
            const uint32_t mw = hmask ? hmask[s >> 5] : ~0u;
            const unsigned long long hv = dig[s];
            if ((mw >> (s & 31)) & 1u) atomicAdd(&h[(uint32_t)(hv >> (64 - b1))], 1u);
        }
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of v over the 256 threads of a block (v of thread t is
// bucket t's count); returns thread t's start.  Uses ws[8] of shared memory.
__device__ __forceinline__ uint32_t pp_block_scan256(uint32_t v, uint32_t* ws) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t pre = 0;
    for (int k = 0; k < w; ++k) pre += ws[k];
    return pre + x - v;
}

// Pairs of a tile in bucket order in shared memory, so that each bucket's
// run is written to global memory contiguously.
constexpr size_t PP_SMEM = (size_t)PP_TILE * (8 + 4);

// Pass 1 scatter: each hashed string's pair to its (bucket, tile) range.
__global__ void __launch_bounds__(PP_NT, 4) k_pp_scatter1(uint64_t n, const unsigned long long* dig,
                                                      const uint32_t* hmask, uint32_t b1, uint32_t ntiles,
                                                      const uint32_t* off, unsigned long long* oh, uint32_t* os) {
    extern __shared__ __align__(16) unsigned char pp_sm[];
    unsigned long long* sh = (unsigned long long*)pp_sm;
    uint32_t* ss = (uint32_t*)(sh + PP_TILE);
    __shared__ uint32_t cnt[256], beg[256], cur[256], gbase[256], ws[8];
    cnt[threadIdx.x] = 0;
    gbase[threadIdx.x] = off[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * PP_TILE;
    // mask words and hashes loaded together, before any is used; a bit of
    // `marked` per position, the bucket recomputed from the hash
    unsigned long long h[PP_IPT];
    uint32_t mw[PP_IPT];
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j) {
        const uint64_t s = t0 + (uint64_t)j * PP_NT + threadIdx.x;
        mw[j] = s < n ? (hmask ? hmask[s >> 5] : ~0u) : 0u;
        h[j] = s < n ? dig[s] : 0ull;
    }
    uint32_t marked = 0;
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j) {
        const uint64_t s = t0 + (uint64_t)j * PP_NT + threadIdx.x;
        if ((mw[j] >> (s & 31)) & 1u) {
            marked |= 1u << j;
            atomicAdd(&cnt[(uint32_t)(h[j] >> (64 - b1))], 1u);
        }
    }
    __syncthreads();
    const uint32_t c = cnt[threadIdx.x];
    const uint32_t e = pp_block_scan256(c, ws);
    beg[threadIdx.x] = e;
    cur[threadIdx.x] = e;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j) {
        if ((marked >> j) & 1u) {
            const uint32_t lp = atomicAdd(&cur[(uint32_t)(h[j] >> (64 - b1))], 1u);
            sh[lp] = h[j];
            ss[lp] = (uint32_t)(t0 + (uint64_t)j * PP_NT + threadIdx.x);
        }
    }
    __syncthreads();
    const uint32_t total = beg[255] + cnt[255];
    for (uint32_t x = threadIdx.x; x < total; x += PP_NT) {
        const unsigned long long hv = sh[x];
        const uint32_t b = (uint32_t)(hv >> (64 - b1));
        const uint32_t dst = gbase[b] + (x - beg[b]);
        oh[dst] = hv;
        os[dst] = ss[x];
    }
}

// Between the passes, one block of 256 threads, thread c for coarse bucket c
// (mid layout: start[256], count[256], first pass-2 tile[257], count base
// [256]): the coarse bucket's range from the pass-1 scan, its pass-2 tiles
// (PP_TILE pairs each) and where its bucket-major counts go.
__global__ void __launch_bounds__(256) k_pp_mid(const uint32_t* off1, uint32_t ntiles1, const uint32_t* total1,
                                               uint32_t b1, uint32_t b2, uint32_t* mid) {
    __shared__ uint32_t sc[256], sh[256];
    const uint32_t c = threadIdx.x;
    const uint32_t nc = 1u << b1;
    uint32_t start = 0, cnt = 0;
    if (c < nc) {
        start = off1[(uint64_t)c * ntiles1];
        cnt = (c + 1 < nc ? off1[(uint64_t)(c + 1) * ntiles1] : *total1) - start;
    }
    const uint32_t nt = (cnt + PP_TILE - 1) / PP_TILE;
    sc[c] = nt;
    sh[c] = nt << b2;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {  // inclusive scans (Hillis-Steele)
        const uint32_t a = c >= (uint32_t)o ? sc[c - o] : 0u, b = c >= (uint32_t)o ? sh[c - o] : 0u;
        __syncthreads();
        sc[c] += a;
        sh[c] += b;
        __syncthreads();
    }
    mid[c] = start;
    mid[256 + c] = cnt;
    mid[512 + c] = sc[c] - nt;
    mid[769 + c] = sh[c] - (nt << b2);
    if (c == 255) mid[512 + 256] = sc[255];
}

__device__ __forceinline__ uint32_t pp_coarse_of(const uint32_t* tile0, uint32_t t) {
    uint32_t lo = 0, hi = 256;  // last c with tile0[c] <= t
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (tile0[m] <= t) lo = m;
        else hi = m;
    }
    return lo;
}

// Pass 2 counts: per tile of a coarse bucket, its pairs per fine bucket (the
// next b2 bits), bucket-major inside the coarse bucket's count block.
__global__ void __launch_bounds__(PP_NT) k_pp_hist2(const unsigned long long* h1, const uint32_t* mid, uint32_t b1,
                                                   uint32_t b2, uint32_t* hist) {
    __shared__ uint32_t h[256], tile0[257];
    const uint32_t t = blockIdx.x;
    if (t >= mid[512 + 256]) return;
    tile0[threadIdx.x] = mid[512 + threadIdx.x];  // searched in shared memory
    if (threadIdx.x == 0) tile0[256] = mid[512 + 256];
    __syncthreads();
    const uint32_t c = pp_coarse_of(tile0, t);
    const uint32_t lt = t - tile0[c], nt = tile0[c + 1] - tile0[c];
    const uint32_t b = mid[c] + lt * PP_TILE, e = mid[c] + min(mid[256 + c], (lt + 1) * PP_TILE);
    h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = b + threadIdx.x; i < e; i += PP_NT) atomicAdd(&h[(uint32_t)((h1[i] << b1) >> (64 - b2))], 1u);
    __syncthreads();
    if (threadIdx.x < (1u << b2)) hist[mid[769 + c] + (uint64_t)threadIdx.x * nt + lt] = h[threadIdx.x];
}

__global__ void __launch_bounds__(PP_NT, 4) k_pp_scatter2(const unsigned long long* h1, const uint32_t* s1,
                                                      const uint32_t* mid, uint32_t b1, uint32_t b2,
                                                      const uint32_t* off, unsigned long long* oh, uint32_t* os) {
    extern __shared__ __align__(16) unsigned char pp_sm[];
    unsigned long long* sh = (unsigned long long*)pp_sm;
    uint32_t* ss = (uint32_t*)(sh + PP_TILE);
    __shared__ uint32_t cnt[256], beg[256], cur[256], gbase[256], ws[8], tile0[257];
    const uint32_t t = blockIdx.x;
    if (t >= mid[512 + 256]) return;
    tile0[threadIdx.x] = mid[512 + threadIdx.x];  // searched in shared memory
    if (threadIdx.x == 0) tile0[256] = mid[512 + 256];
    __syncthreads();
    const uint32_t c = pp_coarse_of(tile0, t);
    const uint32_t lt = t - tile0[c], nt = tile0[c + 1] - tile0[c];
    const uint32_t b = mid[c] + lt * PP_TILE, e = mid[c] + min(mid[256 + c], (lt + 1) * PP_TILE);
    cnt[threadIdx.x] = 0;
    gbase[threadIdx.x] = threadIdx.x < (1u << b2) ? off[mid[769 + c] + (uint64_t)threadIdx.x * nt + lt] : 0u;
    __syncthreads();
    // hashes and strings loaded together, before any is used; the fine
    // bucket recomputed from the hash
    unsigned long long h[PP_IPT];
    uint32_t sv[PP_IPT];
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j) {
        const uint32_t i = b + j * PP_NT + threadIdx.x;
        h[j] = i < e ? h1[i] : 0ull;
        sv[j] = i < e ? s1[i] : 0u;
    }
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j)
        if (b + j * PP_NT + threadIdx.x < e) atomicAdd(&cnt[(uint32_t)((h[j] << b1) >> (64 - b2))], 1u);
    __syncthreads();
    const uint32_t cv = cnt[threadIdx.x];
    const uint32_t ex = pp_block_scan256(cv, ws);
    beg[threadIdx.x] = ex;
    cur[threadIdx.x] = ex;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PP_IPT; ++j) {
        if (b + j * PP_NT + threadIdx.x < e) {
            const uint32_t lp = atomicAdd(&cur[(uint32_t)((h[j] << b1) >> (64 - b2))], 1u);
            sh[lp] = h[j];
            ss[lp] = sv[j];
        }
    }
    __syncthreads();
    const uint32_t total = e - b;
    for (uint32_t x = threadIdx.x; x < total; x += PP_NT) {
        const unsigned long long hv = sh[x];
        const uint32_t f2 = (uint32_t)((hv << b1) >> (64 - b2));
        const uint32_t dst = gbase[f2] + (x - beg[f2]);
        oh[dst] = hv;
        os[dst] = ss[x];
    }
}

// Start of every fine bucket f = (coarse c, fine f2) and the end at [nb].
// With b2 = 0 the coarse buckets are the fine ones.
__global__ void k_pp_starts(const uint32_t* off1, uint32_t ntiles1, const uint32_t* total1, const uint32_t* mid,
                            const uint32_t* off2, uint32_t b2, uint32_t nb, uint32_t* fstart) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f > nb) return;
    if (f == nb) {
        fstart[f] = *total1;
    } else if (b2 == 0) {
        fstart[f] = off1[(uint64_t)f * ntiles1];
    } else {
        const uint32_t c = f >> b2, f2 = f & ((1u << b2) - 1u);
        const uint32_t nt = mid[512 + c + 1] - mid[512 + c];
        fstart[f] = nt ? off2[mid[769 + c] + (uint64_t)f2 * nt] : mid[c];
    }
}

// One block per bucket: every pair whose hash occurs again in the bucket
// (in the same string set) has its string marked in dmask.
__global__ void __launch_bounds__(PD_NT) k_dp_bucket_dups(const uint32_t* fstart, const unsigned long long* ph,
                                                          const uint32_t* ps, uint32_t* dmask, uint32_t* ndup,
                                                          const uint64_t* set_begin, uint32_t nsets,
                                                          uint32_t* overflow) {
    extern __shared__ __align__(16) unsigned char pd_sm[];
    unsigned long long* key = (unsigned long long*)pd_sm;
    uint32_t* tab = (uint32_t*)(key + PD_CAP);
    uint8_t* dup = (uint8_t*)(tab + PD_TAB);
    const uint32_t b = blockIdx.x;
    const uint32_t m = fstart[b + 1] - fstart[b];
    if (m > PD_CAP) {  // the same for the whole block
        if (threadIdx.x == 0) atomicExch(overflow, 1u);
        return;
    }
    const unsigned long long* bh = ph + fstart[b];
    const uint32_t* bs = ps + fstart[b];
    for (uint32_t j = threadIdx.x; j < m; j += PD_NT) {
        key[j] = bh[j];
        dup[j] = 0;
    }
    for (uint32_t j = threadIdx.x; j < PD_TAB; j += PD_NT) tab[j] = 0xFFFFFFFFu;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < m; j += PD_NT) {
        const unsigned long long h = key[j];
        uint32_t sl = (uint32_t)(h ^ (h >> 29)) & (PD_TAB - 1);
        for (uint32_t probe = 0; probe < PD_TAB; ++probe) {
            const uint32_t prev = atomicCAS(&tab[sl], 0xFFFFFFFFu, j);
            if (prev == 0xFFFFFFFFu) break;
            if (key[prev] == h &&
                (nsets <= 1 || set_of(set_begin, nsets, bs[prev]) == set_of(set_begin, nsets, bs[j]))) {
                dup[j] = 1;
                dup[prev] = 1;
                break;
            }
            sl = (sl + 1) & (PD_TAB - 1);
        }
    }
    __syncthreads();
    uint32_t c = 0;
    for (uint32_t j = threadIdx.x; j < m; j += PD_NT) {
        if (dup[j]) {
            const uint32_t s = bs[j];
            atomicOr(&dmask[s >> 5], 1u << (s & 31));
            ++c;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULLM, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(ndup, c);
}

// The owner of every shared slot joins dmask (nothing to do when no insert
// met its own hash).  slots is a multiple of 4: tdup is read a word at a time.
__global__ void __launch_bounds__(256) k_dp_owner_dups(const uint32_t* tdup_words, const uint32_t* tid, uint64_t words,
                                                       uint32_t* dmask, const uint32_t* ndup) {
    if (*ndup == 0) return;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
        const uint32_t v = tdup_words[w];
        if (!v) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b)
            if ((v >> (8 * b)) & 0xFFu) {
                const uint32_t s = tid[4 * w + b];
                atomicOr(&dmask[s >> 5], 1u << (s & 31));
            }
    }
}

// Kind-2 positions whose string's hash is shared stay candidates.
__global__ void __launch_bounds__(256) k_dp_query_mask(const uint8_t* kind, const uint32_t* order,
                                                       const uint32_t* dmask, uint64_t n, uint8_t* st_next,
                                                       uint32_t* counters, const uint32_t* ndup) {
    if (*ndup == 0) return;
    uint32_t nstays = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (kind[i] == 2) {
            const bool stays = bit_of(dmask, order[i]);
            st_next[i] = stays ? 1 : 0;
            nstays += stays;
        }
    }
    block_add(counters + 1, nstays);
}

// Kind-2 positions whose hash was inserted twice stay candidates.  Nothing to
// do when no insert of the round met its own hash (ndup == 0): classification
// already left every kind-2 position retired.
__global__ void __launch_bounds__(256) k_dp_query(const uint8_t* kind, const uint32_t* slot, const uint8_t* tdup,
                                                  uint64_t n, uint8_t* st_next, uint32_t* counters,
                                                  const uint32_t* ndup) {
    if (*ndup == 0) return;
    uint32_t nstays = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (kind[i] == 2) {
            const uint32_t sl = slot[i];
            const bool stays = sl != NO_SLOT && tdup[sl];
            st_next[i] = stays ? 1 : 0;
            nstays += stays;
        }
    }
    block_add(counters + 1, nstays);
}

__global__ void k_prefix_hash(ArenaDev a, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    uint64_t off;
    uint32_t L;
    str_of(a, ids[j], off, L);
    out[j] = filter_hash(xxh64_dev(a.chars + off, depth < L ? depth : L));
}

// Power-of-two table with at least dp_table (>= 2) slots per key: linear
// probing stays short (about 1.5 probes per insert at 2, 1.2 at 4).
static uint64_t table_slots(uint64_t n) {
    const uint64_t k = (uint64_t)tune(TUNE_DP_TABLE);
    uint64_t t = 1024;
    while (t < k * n + 2) t <<= 1;
    return t;
}

// Per-set table regions, the same rule with 64 slots at least (none for a set
// that hashes nothing).  Total <= 3 * hashed + 68 * nsets.
__device__ __forceinline__ uint64_t set_slots(uint32_t c) {
    if (c == 0) return 0;
    uint64_t t = 64;
    while (t < (uint64_t)c + c / 2 + 2) t <<= 1;
    return t;
}

// Per-set filter regions in 32-bit words: a power of two >= bpk bits per
// hashed string, 1024 bits at least.
__device__ __forceinline__ uint64_t set_filter_bits(uint32_t c, uint32_t bpk) {
    if (c == 0) return 0;
    uint64_t t = 1024;
    while (t < (uint64_t)c * bpk) t <<= 1;
    return t;
}

constexpr int SET_NT = 1024;

// One block: region base and mask per set from the per-set counts, total into
// out[0..1] (lo, hi), *err set if it exceeds cap.  bpk == 0: hash-table
// regions (slots); bpk > 0: filter regions (base in words, mask in bits).
__global__ void __launch_bounds__(SET_NT) k_set_tables(const uint32_t* cnt, uint32_t nsets, uint64_t cap, uint32_t bpk,
                                                       uint64_t* base, uint32_t* mask, uint32_t* out, uint32_t* err) {
    __shared__ uint64_t part[SET_NT];
    const uint32_t per = (nsets + SET_NT - 1) / SET_NT;
    const uint32_t b = min(nsets, threadIdx.x * per), e = min(nsets, b + per);
    auto size_of = [&](uint32_t c) -> uint64_t { return bpk ? set_filter_bits(c, bpk) / 32 : set_slots(c); };
    uint64_t sum = 0;
    for (uint32_t s = b; s < e; ++s) sum += size_of(cnt[s]);
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < SET_NT; off <<= 1) {
        const uint64_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint64_t run = part[threadIdx.x] - sum;
    for (uint32_t s = b; s < e; ++s) {
        const uint64_t sl = size_of(cnt[s]);
        base[s] = run;
        mask[s] = sl ? (uint32_t)((bpk ? sl * 32 : sl) - 1) : 0;
        run += sl;
    }
    if (threadIdx.x == SET_NT - 1) {
        const uint64_t total = part[SET_NT - 1];
        if (total > cap) *err = 1;
        out[0] = (uint32_t)total;
        out[1] = (uint32_t)(total >> 32);
    }
}

// ---------------------------------------------------- fingerprint filter ----
// Rounds that hash many strings find duplicate hashes without a table entry
// per string: each hashed string sets one bit, chosen by its hash, of a
// bitmap small enough to stay in L2; a string whose bit was already set is a
// candidate.  Every hash that occurs twice has a candidate (its later insert),
// so an exact table over the candidates' hashes, in which every hashed string
// then counts itself if its hash is there, gives the exact number of strings
// per duplicated hash; a string whose hash is not in that table is unique.
// The outcome is exactly that of one table over all hashes.
__global__ void k_dp_filter(ArenaDev a, const uint64_t* soff, const uint8_t* kind, uint64_t n, uint32_t depth,
                            uint32_t* bits, uint32_t bmask1, const uint64_t* set_begin, uint32_t nsets,
                            const uint64_t* set_wbase, const uint32_t* set_bmask, unsigned long long* hbuf,
                            uint32_t* cand, uint32_t* ncand, uint32_t* set_ccnt) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool c = false;
    uint32_t sid = 0;
    if (i < n && kind[i] >= 2) {
        const unsigned long long h = filter_hash(xxh64_dev(a.chars + soff[i], depth));
        hbuf[i] = h;
        uint64_t wbase = 0;
        uint32_t bm = bmask1;
        if (nsets > 1) {
            sid = set_of(set_begin, nsets, i);
            wbase = set_wbase[sid];
            bm = set_bmask[sid];
        }
        const uint32_t b = (uint32_t)(h >> 32) & bm;
        const uint32_t bit = 1u << (b & 31);
        c = (atomicOr(&bits[wbase + (b >> 5)], bit) & bit) != 0;
    }
    const int lane = threadIdx.x & 31;
    const uint32_t m = __ballot_sync(FULLM, c);
    if (m) {
        uint32_t base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(ncand, (uint32_t)__popc(m));
        base = __shfl_sync(FULLM, base, __ffs(m) - 1);
        if (c) cand[base + __popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
        if (nsets > 1) {
            const uint32_t key = c ? sid : 0xFFFFFFFFu - lane;
            const uint32_t peers = __match_any_sync(FULLM, key);
            if (c && lane == __ffs(peers) - 1) atomicAdd(&set_ccnt[sid], (uint32_t)__popc(peers));
        }
    }
}

// Table region of position i: (base, mask).
__device__ __forceinline__ void table_region(const uint64_t* set_begin, uint32_t nsets, const uint64_t* set_base,
                                             const uint32_t* set_mask, uint32_t mask1, uint64_t i, uint64_t& base,
                                             uint32_t& mask) {
    base = 0;
    mask = mask1;
    if (nsets > 1) {
        const uint32_t sid = set_of(set_begin, nsets, i);
        base = set_base[sid];
        mask = set_mask[sid];
    }
}

// Inserts the candidates' hashes (each distinct hash once).
__global__ void k_cand_insert(const uint32_t* cand, uint32_t ncand, const unsigned long long* hbuf,
                              unsigned long long* tkeys, uint32_t mask1, const uint64_t* set_begin, uint32_t nsets,
                              const uint64_t* set_base, const uint32_t* set_mask, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ncand) return;
    const uint32_t i = cand[j];
    const unsigned long long h = hbuf[i];
    uint64_t base;
    uint32_t mask;
    table_region(set_begin, nsets, set_base, set_mask, mask1, i, base, mask);
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    for (uint32_t probe = 0;; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            return;
        }
        const unsigned long long prev = atomicCAS(&tkeys[base + sl], EMPTY_KEY, h);
        if (prev == EMPTY_KEY || prev == h) return;
        sl = (sl + 1) & mask;
    }
}

// Every hashed string whose hash is in the candidate table counts itself
// there: tcnt byte bit 0 = seen, bit 1 = seen twice or more.
__global__ void k_dp_count(const uint8_t* kind, uint64_t n, const unsigned long long* hbuf,
                           const unsigned long long* tkeys, uint32_t* tcnt_words, uint32_t mask1,
                           const uint64_t* set_begin, uint32_t nsets, const uint64_t* set_base,
                           const uint32_t* set_mask, uint32_t* slot, uint32_t* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] < 2) return;
    const unsigned long long h = hbuf[i];
    uint64_t base;
    uint32_t mask;
    table_region(set_begin, nsets, set_base, set_mask, mask1, i, base, mask);
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    uint32_t found = NO_SLOT;
    // a set without candidates has no region (mask 0): nothing to find
    for (uint32_t probe = 0; mask != 0; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            break;
        }
        const unsigned long long k = tkeys[base + sl];
        if (k == h) {
            found = (uint32_t)(base + sl);
            break;
        }
        if (k == EMPTY_KEY) break;
        sl = (sl + 1) & mask;
    }
    slot[i] = found;
    if (found != NO_SLOT) {
        const uint32_t sh = 8 * (found & 3u);
        const uint32_t old = atomicOr(&tcnt_words[found >> 2], 1u << sh);
        if (old & (1u << sh)) atomicOr(&tcnt_words[found >> 2], 2u << sh);
    }
}

__global__ void k_dp_query_cnt(const uint8_t* kind, const uint32_t* slot, const uint8_t* tcnt, uint64_t n,
                               uint8_t* st_next, uint32_t* counters) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool stays = false;
    if (i < n && kind[i] == 2) {
        const uint32_t sl = slot[i];
        stays = sl != NO_SLOT && (tcnt[sl] & 2);
        st_next[i] = stays ? 1 : 0;
    }
    block_count(counters + 1, stays);
}

static uint64_t pow2_at_least(uint64_t x, uint64_t lo) {
    uint64_t t = lo;
    while (t < x) t <<= 1;
    return t;
}

void layout_dp(Carve& c, DpLayout& L, uint64_t n, uint32_t nsets) {
    uint64_t N = n ? n : 1;
    if (nsets == 0) nsets = 1;
    L.nsets_cap = nsets;
    L.set_begin = c.take<uint64_t>(nsets + 1);
    L.set_base = c.take<uint64_t>(nsets + 1);
    L.set_mask = c.take<uint32_t>(nsets);
    L.set_cnt = c.take<uint32_t>(nsets);
    L.st[0] = c.take<uint8_t>(N);
    L.st[1] = c.take<uint8_t>(N);
    L.kind = c.take<uint8_t>(N);
    L.lens = c.take<uint32_t>(N);
    L.soff = c.take<uint64_t>(N);
    L.minlen = c.take<uint32_t>(2);  // shortest string, smallest neighbour LCP
    L.slot = c.take<uint32_t>(N);
    // one set: the table for n keys; several: room for every set's own
    // power-of-two region (at most 3 slots per key plus 68 per set)
    L.slots = nsets == 1 ? table_slots(N) : 3 * N + 128ull * (nsets + 1);
    L.tkeys = c.take<unsigned long long>(L.slots);
    L.tdup = c.take<uint8_t>(L.slots + 4);
    L.counters = c.take<uint32_t>(16);
    L.set_bbase = c.take<uint64_t>(nsets);
    L.set_bmask = c.take<uint32_t>(nsets);
    L.set_ccnt = c.take<uint32_t>(nsets);
    // fingerprint filter: planned when a round may hash dp_filter_min strings
    L.filter_min = (uint64_t)tune(TUNE_DP_FILTER_MIN);
    L.filter_bpk = (uint32_t)tune(TUNE_DP_FILTER_BITS);
    L.split = tune(TUNE_DP_SPLIT) != 0;
    // arena-order hashes for dense rounds (every string of the arena)
    L.digest_share = (uint32_t)tune(TUNE_DP_DIGEST);
    L.mask_words = (N + 31) / 32;
    L.hmask = L.digest_share ? c.take<uint32_t>(L.mask_words) : nullptr;
    L.dmask = L.digest_share ? c.take<uint32_t>(L.mask_words) : nullptr;
    L.tid = L.digest_share ? c.take<uint32_t>(L.slots) : nullptr;
    // bucket regions of the dense rounds (at most pd_buckets(N) buckets)
    L.pd_nb = L.digest_share ? std::max<uint32_t>(pd_buckets(N), 2) : 0;
    if (L.digest_share) {
        L.pd_start = c.take<uint32_t>(L.pd_nb + 1);
        L.pd_h = c.take<unsigned long long>(N);
        L.pd_s = c.take<uint32_t>(N);
        L.pp_h1 = c.take<unsigned long long>(N);
        L.pp_s1 = c.take<uint32_t>(N);
        L.pp_dig = c.take<unsigned long long>(N);
        // pass-1 counts: 256 per tile of positions; pass 2: at most 256 per
        // tile of pairs plus one partial tile per coarse bucket
        L.pp_hcap = 256ull * ((N + PP_TILE - 1) / PP_TILE + 257);
        L.pp_hist = c.take<uint32_t>(L.pp_hcap);
        L.pp_off = c.take<uint32_t>(2 * L.pp_hcap);
        L.pp_mid = c.take<uint32_t>(1032);
        L.pp_total = c.take<uint32_t>(4);
        L.pp_scan = c.take<unsigned char>(scan_scratch_bytes(L.pp_hcap));
    } else {
        L.pd_start = nullptr;
        L.pd_h = nullptr;
        L.pd_s = nullptr;
        L.pp_h1 = nullptr;
        L.pp_s1 = nullptr;
        L.pp_dig = nullptr;
        L.pp_hcap = 0;
        L.pp_hist = nullptr;
        L.pp_off = nullptr;
        L.pp_mid = nullptr;
        L.pp_total = nullptr;
        L.pp_scan = nullptr;
    }
    const bool filter = N >= L.filter_min;
    L.hbuf = (filter || L.split) ? c.take<unsigned long long>(N) : nullptr;
    if (filter) {
        L.bm_words = (nsets == 1 ? pow2_at_least(N * L.filter_bpk, 1024) : 2 * N * L.filter_bpk + 1024ull * nsets) / 32;
        L.bits = c.take<uint32_t>(L.bm_words);
        L.cand = c.take<uint32_t>(N);
    } else {
        L.bm_words = 0;
        L.bits = nullptr;
        L.cand = nullptr;
    }
}

int dp_rounds(const DpLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
              uint32_t* dp, uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds, uint32_t* pin,
              cudaStream_t st, uint32_t nsets, const uint64_t* set_begin_host, const unsigned long long* rdig,
              uint32_t rdig_mask) {
    uint32_t r = 0;
    if (n == 0) {
        if (rounds) *rounds = 0;
        return DSSS_OK;
    }
    if (nsets == 0) nsets = 1;
    if (nsets > 1) {
        if (!set_begin_host || nsets > L.nsets_cap) return fail(DSSS_EINVAL, "string sets not planned");
        DSSS_CUDA(cudaMemcpyAsync(L.set_begin, set_begin_host, (nsets + 1) * sizeof(uint64_t),
                                  cudaMemcpyHostToDevice, st));
    }
    const unsigned grid = grid_for(n, 256);
    // lengths and offsets in sorted order are gathered (k_dp_lens, one random
    // handle read per position) only once a round needs them: a depth past
    // the shortest string of the arena, or hashes taken in sorted order
    DSSS_CUDA(cudaMemsetAsync(L.minlen, 0xFF, 2 * sizeof(uint32_t), st));
    DSSS_LAUNCH("k_min_len", st,
                k_min_len<<<(unsigned)std::min<uint64_t>(grid_for(a.n, 256), 148 * 8), 256, 0, st>>>(
                    a.len, a.h, a.n, L.minlen));
    DSSS_LAUNCH("k_min_nbr_lcp", st,
                k_min_nbr_lcp<<<(unsigned)std::min<uint64_t>(grid_for(n, 256), 148 * 8), 256, 0, st>>>(lcp, n,
                                                                                                      L.minlen + 1));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.minlen, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    const uint64_t min_len = pin[0];
    // rounds up to this depth, while every string is a candidate, keep every
    // string and are not run (their candidate counts are recorded as n)
    const uint64_t trivial_to = std::min<uint64_t>(min_len, pin[1]);
    bool all_cands = true;
    bool lens_ready = false;
    auto need_lens = [&]() -> int {
        if (!lens_ready) {
            DSSS_LAUNCH("k_dp_lens", st, k_dp_lens<<<lens_grid(n), 256, 0, st>>>(a, order, n, L.lens, L.soff));
            lens_ready = true;
        }
        return DSSS_OK;
    };
    int cur = 0;
    const uint64_t start = 8;
    uint64_t depth = start;
    uint64_t cands = n;  // candidates entering the round
    for (uint64_t i = start * 2;; i *= 2) {
        if (depth > 0xFFFFFFFFull) return fail(DSSS_EINVAL, "distinguishing-prefix depth overflow");
        if (all_cands && depth <= trivial_to) {
            if (round_counts && r < max_rounds) round_counts[r] = n;
            ++r;
            depth = start + i;
            continue;
        }
        DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 16 * sizeof(uint32_t), st));
        if (nsets > 1) DSSS_CUDA(cudaMemsetAsync(L.set_cnt, 0, nsets * sizeof(uint32_t), st));
        // a round that may turn out dense marks its hashed strings for the
        // arena-order form (every string of the arena must be in the order)
        const bool mark = L.hmask && a.n <= n && cands * L.digest_share >= n;
        // the hashed strings are marked after the count, only when not every
        // string of the arena is hashed (a null mask then stands for all)
        uint32_t* hm = nullptr;
        if (depth > min_len) DSSS_TRY(need_lens());
        const uint32_t* lens = lens_ready ? L.lens : nullptr;  // nullptr: every string reaches the depth
        if (nsets == 1 && aligned16(lcp) && aligned16(dp) && aligned16(L.lens) && aligned16(L.st[cur]) &&
            aligned16(L.st[cur ^ 1]) && aligned16(L.kind)) {
            DSSS_LAUNCH("k_dp_classify", st,
                        k_dp_classify4<<<stride_grid((n + 3) / 4), 256, 0, st>>>(L.st[cur], all_cands, lens, lcp, n,
                                                                                (uint32_t)depth, dp, L.st[cur ^ 1],
                                                                                L.kind, L.counters, order, hm));
        } else {
            DSSS_LAUNCH("k_dp_classify", st,
                        k_dp_classify<<<stride_grid(n), 256, 0, st>>>(L.st[cur], all_cands, lens, lcp, n, (uint32_t)depth,
                                                                     dp, L.st[cur ^ 1], L.kind, L.counters,
                                                                     L.set_begin, nsets, L.set_cnt, order, hm));
        }
        if (nsets > 1) {
            DSSS_LAUNCH("k_set_tables", st,
                        k_set_tables<<<1, SET_NT, 0, st>>>(L.set_cnt, nsets, L.slots, 0, L.set_base, L.set_mask,
                                                           L.counters + 4, L.counters + 2));
            if (L.bits)
                DSSS_LAUNCH("k_set_tables", st,
                            k_set_tables<<<1, SET_NT, 0, st>>>(L.set_cnt, nsets, L.bm_words, L.filter_bpk,
                                                               L.set_bbase, L.set_bmask, L.counters + 6,
                                                               L.counters + 2));
        }
        DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        const uint32_t hashed = pin[0];
        if (pin[2]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table regions exceed the plan");
        if (hashed && L.bits && hashed >= L.filter_min) {
            // fingerprint filter, then an exact table over the candidates only
            DSSS_TRY(need_lens());
            const uint64_t words = nsets > 1 ? ((uint64_t)pin[7] << 32 | pin[6])
                                             : pow2_at_least((uint64_t)hashed * L.filter_bpk, 1024) / 32;
            if (words > L.bm_words) return fail(DSSS_EDEVICE, "distinguishing-prefix filter exceeds the plan");
            DSSS_CUDA(cudaMemsetAsync(L.bits, 0, words * 4, st));
            if (nsets > 1) DSSS_CUDA(cudaMemsetAsync(L.set_ccnt, 0, nsets * sizeof(uint32_t), st));
            DSSS_LAUNCH("k_dp_filter", st,
                        k_dp_filter<<<grid, 256, 0, st>>>(a, L.soff, L.kind, n, (uint32_t)depth, L.bits,
                                                         (uint32_t)(words * 32 - 1), L.set_begin, nsets, L.set_bbase,
                                                         L.set_bmask, L.hbuf, L.cand, L.counters + 3, L.set_ccnt));
            if (nsets > 1)
                DSSS_LAUNCH("k_set_tables", st,
                            k_set_tables<<<1, SET_NT, 0, st>>>(L.set_ccnt, nsets, L.slots, 0, L.set_base, L.set_mask,
                                                               L.counters + 4, L.counters + 2));
            DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaStreamSynchronize(st));
            if (pin[2]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table regions exceed the plan");
            const uint32_t ncand = pin[3];
            if (ncand) {  // else every hash is unique: no kind-2 string stays
                const uint64_t slots = nsets > 1 ? ((uint64_t)pin[5] << 32 | pin[4]) : table_slots(ncand);
                if (slots > L.slots) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table exceeds the plan");
                DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
                DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, (slots + 3) & ~3ull, st));
                DSSS_LAUNCH("k_cand_insert", st,
                            k_cand_insert<<<grid_for(ncand, 256), 256, 0, st>>>(L.cand, ncand, L.hbuf, L.tkeys,
                                                                                 (uint32_t)(slots - 1), L.set_begin,
                                                                                 nsets, L.set_base, L.set_mask,
                                                                                 L.counters + 2));
                DSSS_LAUNCH("k_dp_count", st,
                            k_dp_count<<<grid, 256, 0, st>>>(L.kind, n, L.hbuf, L.tkeys, (uint32_t*)L.tdup,
                                                            (uint32_t)(slots - 1), L.set_begin, nsets, L.set_base,
                                                            L.set_mask, L.slot, L.counters + 2));
                DSSS_LAUNCH("k_dp_query", st,
                            k_dp_query_cnt<<<grid, 256, 0, st>>>(L.kind, L.slot, L.tdup, n, L.st[cur ^ 1],
                                                                L.counters));
                DSSS_CUDA(cudaGetLastError());
                DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                DSSS_CUDA(cudaStreamSynchronize(st));
                if (pin[2]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table overflow");
            }
        } else if (hashed) {
            const uint64_t slots = nsets > 1 ? ((uint64_t)pin[5] << 32 | pin[4]) : table_slots(hashed);
            if (slots > L.slots) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table exceeds the plan");
            const bool arena = mark && (uint64_t)hashed * L.digest_share >= n;
            const uint32_t check = (uint32_t)tune(TUNE_DP_CHECK);
            const uint32_t* hmask = nullptr;  // every string of the arena hashed
            if (arena && hashed < a.n) {
                DSSS_CUDA(cudaMemsetAsync(L.hmask, 0, L.mask_words * sizeof(uint32_t), st));
                DSSS_LAUNCH("k_dp_mark", st,
                            k_dp_mark<<<grid_for(n, 256), 256, 0, st>>>(L.kind, order, n, L.hmask));
                hmask = L.hmask;
            }
            if (arena) {
                const int dj = root_digest_index(depth);
                const unsigned long long* dig =
                    rdig && dj >= 0 && ((rdig_mask >> dj) & 1u) ? rdig + (uint64_t)dj * a.n : nullptr;
                // buckets in shared memory first; the table only if a bucket overflows
                bool done = false;
                uint32_t bbits = 1;  // at least two buckets (both radix shifts stay below 64)
                while ((1ull << bbits) < pd_buckets(hashed)) ++bbits;
                const uint32_t nb = 1u << bbits;
                if (nb <= L.pd_nb && bbits <= 16) {
                    static std::atomic<uint64_t> pd_configured{0};
                    DSSS_TRY(set_smem_once(pd_configured, k_dp_bucket_dups, (int)PD_SMEM));
                    DSSS_CUDA(cudaMemsetAsync(L.dmask, 0, L.mask_words * sizeof(uint32_t), st));
                    const unsigned long long* hd = dig;
                    if (!dig || check) {  // this round's hashes, in arena order
                        DSSS_LAUNCH("k_dp_arena_hash", st,
                                    k_dp_arena_hash<<<grid_for(a.n, 256), 256, 0, st>>>(
                                        a, (uint32_t)depth, check ? dig : nullptr, hmask, L.pp_dig, L.counters + 9));
                        hd = L.pp_dig;
                    }
                    // two radix passes: top b1 bits, then the next b2 inside each coarse bucket
                    const uint32_t b1 = std::min<uint32_t>(bbits, 8), b2 = bbits - b1;
                    const uint32_t nt1 = (uint32_t)((a.n + PP_TILE - 1) / PP_TILE);
                    DSSS_LAUNCH("k_pp_hist1", st,
                                k_pp_hist1<<<nt1, PP_NT, 0, st>>>(a.n, hd, hmask, b1, nt1, L.pp_hist));
                    DSSS_TRY(exclusive_scan_u32(L.pp_hist, L.pp_off, 256ull * nt1, L.pp_total, L.pp_scan, st));
                    const unsigned long long* ph = L.pp_h1;
                    const uint32_t* ps = L.pp_s1;
                    static std::atomic<uint64_t> pp1_configured{0}, pp2_configured{0};
                    DSSS_TRY(set_smem_once(pp1_configured, k_pp_scatter1, (int)PP_SMEM));
                    DSSS_TRY(set_smem_once(pp2_configured, k_pp_scatter2, (int)PP_SMEM));
                    DSSS_LAUNCH("k_pp_scatter1", st,
                                k_pp_scatter1<<<nt1, PP_NT, PP_SMEM, st>>>(a.n, hd, hmask, b1, nt1, L.pp_off, L.pp_h1,
                                                                           L.pp_s1));
                    uint32_t* off2 = nullptr;
                    if (b2) {
                        // pass-2 tiles: at most one partial tile per coarse bucket beyond hashed / PP_TILE
                        const uint64_t nt2 = hashed / PP_TILE + 257;
                        const uint64_t h2 = nt2 << b2;
                        if (h2 > L.pp_hcap) return fail(DSSS_EDEVICE, "distinguishing-prefix partition exceeds the plan");
                        off2 = L.pp_off + L.pp_hcap;  // the second pass's offsets beside the first's
                        DSSS_LAUNCH("k_pp_mid", st,
                                    k_pp_mid<<<1, 256, 0, st>>>(L.pp_off, nt1, L.pp_total, b1, b2, L.pp_mid));
                        DSSS_CUDA(cudaMemsetAsync(L.pp_hist, 0, h2 * sizeof(uint32_t), st));
                        DSSS_LAUNCH("k_pp_hist2", st,
                                    k_pp_hist2<<<(unsigned)nt2, PP_NT, 0, st>>>(L.pp_h1, L.pp_mid, b1, b2, L.pp_hist));
                        DSSS_TRY(exclusive_scan_u32(L.pp_hist, off2, h2, L.pp_total + 1, L.pp_scan, st));
                        DSSS_LAUNCH("k_pp_scatter2", st,
                                    k_pp_scatter2<<<(unsigned)nt2, PP_NT, PP_SMEM, st>>>(L.pp_h1, L.pp_s1, L.pp_mid, b1,
                                                                                         b2, off2, L.pd_h, L.pd_s));
                        ph = L.pd_h;
                        ps = L.pd_s;
                    }
                    DSSS_LAUNCH("k_pp_starts", st,
                                k_pp_starts<<<grid_for(nb + 1, 256), 256, 0, st>>>(L.pp_off, nt1, L.pp_total, L.pp_mid,
                                                                                  off2, b2, nb, L.pd_start));
                    DSSS_LAUNCH("k_dp_bucket_dups", st,
                                k_dp_bucket_dups<<<nb, PD_NT, PD_SMEM, st>>>(L.pd_start, ph, ps, L.dmask,
                                                                            L.counters + 8, L.set_begin, nsets,
                                                                            L.counters + 10));
                    DSSS_CUDA(cudaGetLastError());
                    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 12 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                    DSSS_CUDA(cudaStreamSynchronize(st));
                    done = pin[10] == 0;
                    if (!done) DSSS_CUDA(cudaMemsetAsync(L.counters + 8, 0, 4 * sizeof(uint32_t), st));
                }
                if (!done) {
                    DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
                    DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, slots, st));
                    DSSS_CUDA(cudaMemsetAsync(L.dmask, 0, L.mask_words * sizeof(uint32_t), st));
                    DSSS_LAUNCH("k_dp_arena_insert", st,
                                k_dp_arena_insert<<<grid_for(a.n, 256), 256, 0, st>>>(
                                    a, (uint32_t)depth, dig, hmask, L.tkeys, L.tdup, L.tid, (uint32_t)(slots - 1),
                                    L.set_begin, nsets, L.set_base, L.set_mask, L.dmask, L.counters + 2,
                                    L.counters + 8, check, L.counters + 9));
                    DSSS_LAUNCH("k_dp_owner_dups", st,
                                k_dp_owner_dups<<<stride_grid(slots / 4), 256, 0, st>>>(
                                    (const uint32_t*)L.tdup, L.tid, slots / 4, L.dmask, L.counters + 8));
                }
                DSSS_LAUNCH("k_dp_query", st,
                            k_dp_query_mask<<<stride_grid(n), 256, 0, st>>>(L.kind, order, L.dmask, n, L.st[cur ^ 1],
                                                                           L.counters, L.counters + 8));
            } else {
                // hashes in sorted order read the offsets: gathered for all
                // positions unless few hash (those find theirs through order)
                if (L.split || !sparse_round(hashed, n)) DSSS_TRY(need_lens());
                DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
                DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, slots, st));
                if (L.split) {
                    DSSS_LAUNCH("k_dp_hash_store", st,
                                k_dp_hash_store<<<grid, 256, 0, st>>>(a, L.soff, L.kind, n, (uint32_t)depth, L.hbuf));
                    DSSS_LAUNCH("k_dp_insert", st,
                                k_dp_insert<<<grid, 256, 0, st>>>(L.kind, n, L.hbuf, L.tkeys, L.tdup,
                                                                 (uint32_t)(slots - 1), L.set_begin, nsets, L.set_base,
                                                                 L.set_mask, L.slot, L.counters + 2, L.counters + 8));
                } else {
                    DSSS_TRY(launch_dp_hash(a, lens_ready ? L.soff : nullptr, order, L.kind, n, (uint32_t)depth, hashed,
                                            L.tkeys, L.tdup,
                                            (uint32_t)(slots - 1), L.set_begin, nsets, L.set_base, L.set_mask, L.slot,
                                            L.counters + 2, L.counters + 8, st));
                }
                DSSS_LAUNCH("k_dp_query", st,
                            k_dp_query<<<stride_grid(n), 256, 0, st>>>(L.kind, L.slot, L.tdup, n, L.st[cur ^ 1],
                                                                      L.counters, L.counters + 8));
            }
            DSSS_CUDA(cudaGetLastError());
            DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 10 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaStreamSynchronize(st));
            if (pin[2]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table overflow");
            if (pin[9]) return fail(DSSS_EDEVICE, "a stored prefix hash differs from the string's (dp_check)");
        }
        const uint32_t m = pin[1];
        if (round_counts && r < max_rounds) round_counts[r] = m;
        ++r;
        cur ^= 1;
        all_cands = false;
        if (m == 0) break;
        cands = m;
        depth = start + i;
    }
    if (rounds) *rounds = r;
    return DSSS_OK;
}

__global__ void k_cand_to_state(const uint32_t* cand, uint64_t m, uint64_t n, uint8_t* st, uint32_t* err) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t i = cand[j];
    if (i >= n || (j > 0 && cand[j - 1] >= i)) {  // positions must be ascending and in range
        atomicExch(err, 1u);
        return;
    }
    st[i] = 1;
}

__global__ void k_state_flags(const uint8_t* st, uint64_t n, uint32_t* flag) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = st[i];
}

__global__ void k_state_compact(const uint32_t* flag, const uint32_t* pos, uint64_t n, uint32_t* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flag[i]) out[pos[i]] = (uint32_t)i;
}

void layout_dp_round(Carve& c, DpRoundLayout& R, uint64_t n) {
    layout_dp(c, R.dp, n);
    const uint64_t N = n ? n : 1;
    R.flag = c.take<uint32_t>(N);
    R.pos = c.take<uint32_t>(N);
    R.total = c.take<uint32_t>(2);
    R.scan = c.take<unsigned char>(scan_scratch_bytes(N));
}

int dp_one_round(const DpRoundLayout& R, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
                 const uint32_t* cand, uint64_t m, uint32_t depth, uint32_t* dp, uint32_t* next, uint64_t* m_next,
                 uint32_t* pin, cudaStream_t st) {
    const DpLayout& L = R.dp;
    *m_next = 0;
    if (n == 0) return DSSS_OK;
    const unsigned grid = grid_for(n, 256);
    DSSS_LAUNCH("k_dp_lens", st, k_dp_lens<<<lens_grid(n), 256, 0, st>>>(a, order, n, L.lens, L.soff));
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 16 * sizeof(uint32_t), st));
    const bool all = cand == nullptr;
    if (!all) {
        DSSS_CUDA(cudaMemsetAsync(L.st[0], 0, n, st));
        if (m) DSSS_LAUNCH("k_cand_to_state", st,
                           k_cand_to_state<<<grid_for(m, 256), 256, 0, st>>>(cand, m, n, L.st[0], L.counters + 3));
    }
    DSSS_LAUNCH("k_dp_classify", st,
                k_dp_classify<<<stride_grid(n), 256, 0, st>>>(L.st[0], all, L.lens, lcp, n, depth, dp, L.st[1], L.kind,
                                                   L.counters, nullptr, 1, nullptr));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[3]) return fail(DSSS_EINVAL, "candidates must be ascending positions below n");
    if (pin[0]) {
        const uint64_t slots = table_slots(pin[0]);
        DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
        DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, slots, st));
        DSSS_TRY(launch_dp_hash(a, L.soff, order, L.kind, n, depth, pin[0], L.tkeys, L.tdup, (uint32_t)(slots - 1), nullptr,
                                1, nullptr, nullptr, L.slot, L.counters + 2, L.counters + 8, st));
        DSSS_LAUNCH("k_dp_query", st,
                    k_dp_query<<<stride_grid(n), 256, 0, st>>>(L.kind, L.slot, L.tdup, n, L.st[1], L.counters,
                                                              L.counters + 8));
    }
    DSSS_LAUNCH("k_state_flags", st, k_state_flags<<<grid, 256, 0, st>>>(L.st[1], n, R.flag));
    DSSS_TRY(exclusive_scan_u32(R.flag, R.pos, n, R.total, R.scan, st));
    DSSS_LAUNCH("k_state_compact", st, k_state_compact<<<grid, 256, 0, st>>>(R.flag, R.pos, n, next));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(pin + 4, R.total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[2]) return fail(DSSS_EDEVICE, "distinguishing-prefix hash table overflow");
    *m_next = pin[4];
    return DSSS_OK;
}

int prefix_hash(const ArenaDev& a, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* out,
                cudaStream_t st) {
    if (m == 0) return DSSS_OK;
    DSSS_LAUNCH("k_prefix_hash", st, k_prefix_hash<<<grid_for(m, 256), 256, 0, st>>>(a, ids, m, depth, out));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

// ------------------------------------------------- PEs on several GPUs ----
// One distinguishing-prefix round split where the hashes cross GPUs: the
// classification and the hashes of this GPU's candidates (dp_classify_hash),
// the duplicate test on the hashes routed to this GPU (hash_route, hash_dups)
// and the outcome applied to the candidate states (dp_apply).

__global__ void k_hash_flags(const uint8_t* kind, uint64_t n, uint32_t* flag) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = kind[i] >= 2 ? 1u : 0u;
}

__global__ void k_hash_compact(ArenaDev a, const uint64_t* soff, const uint8_t* kind, const uint32_t* pos, uint64_t n,
                               uint32_t depth, uint32_t* hpos, unsigned long long* hval) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] < 2) return;
    const uint32_t j = pos[i];
    hpos[j] = (uint32_t)i;
    hval[j] = filter_hash(xxh64_dev(a.chars + soff[i], depth));
}

void layout_dp_split(Carve& c, DpSplitLayout& L, uint64_t n) {
    const uint64_t N = n ? n : 1;
    L.lens = c.take<uint32_t>(N);
    L.soff = c.take<uint64_t>(N);
    L.kind = c.take<uint8_t>(N);
    L.flag = c.take<uint32_t>(N);
    L.pos = c.take<uint32_t>(N);
    L.counters = c.take<uint32_t>(16);
    L.scan = c.take<unsigned char>(scan_scratch_bytes(N));
}

int dp_classify_hash(const DpSplitLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
                     const uint8_t* state_in, uint32_t depth, uint32_t* dp, uint8_t* state_out, uint32_t* hpos,
                     unsigned long long* hval, uint64_t* m, uint32_t* pin, cudaStream_t st) {
    *m = 0;
    if (n == 0) return DSSS_OK;
    const unsigned grid = grid_for(n, 256);
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 16 * sizeof(uint32_t), st));
    DSSS_LAUNCH("k_dp_lens", st, k_dp_lens<<<lens_grid(n), 256, 0, st>>>(a, order, n, L.lens, L.soff));
    DSSS_LAUNCH("k_dp_classify", st,
                k_dp_classify<<<stride_grid(n), 256, 0, st>>>(state_in, state_in == nullptr, L.lens, lcp, n, depth, dp, state_out,
                                                   L.kind, L.counters, nullptr, 1, nullptr));
    DSSS_LAUNCH("k_hash_flags", st, k_hash_flags<<<grid, 256, 0, st>>>(L.kind, n, L.flag));
    DSSS_TRY(exclusive_scan_u32(L.flag, L.pos, n, L.counters + 4, L.scan, st));
    DSSS_LAUNCH("k_hash_compact", st,
                k_hash_compact<<<grid, 256, 0, st>>>(a, L.soff, L.kind, L.pos, n, depth, hpos, hval));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    *m = pin[4];
    return DSSS_OK;
}

// Owner of a hash among nowner GPUs: equal slices of the 64-bit range.
__device__ __forceinline__ uint32_t hash_owner(unsigned long long h, uint32_t nowner) {
    return (uint32_t)__umul64hi(h, (unsigned long long)nowner);
}

__global__ void k_hash_owner(const unsigned long long* hval, uint64_t m, uint32_t nowner, uint32_t* owner,
                             unsigned long long* counts) {
    extern __shared__ uint32_t hcnt[];
    for (uint32_t k = threadIdx.x; k < nowner; k += blockDim.x) hcnt[k] = 0;
    __syncthreads();
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t o = hash_owner(hval[j], nowner);
        owner[j] = o;
        atomicAdd(&hcnt[o], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nowner; k += blockDim.x)
        if (hcnt[k]) atomicAdd(&counts[k], (unsigned long long)hcnt[k]);
}

__global__ void k_route_scatter(const unsigned long long* hval, const uint32_t* hpos, const uint32_t* dest, uint64_t m,
                                unsigned long long* out_hval, uint32_t* out_hpos) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t d = dest[j];
    out_hval[d] = hval[j];
    out_hpos[d] = hpos[j];
}

// Hash records in hash order (ips4o::sort of the round's HashStringIndex
// records, bloomfilter.hpp:1512): a stable LSD radix sort, eight passes of
// one byte, each a stable multisplit of the records by that byte.
__global__ void k_hash_byte(const unsigned long long* h, uint64_t m, uint32_t shift, uint32_t* dig) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) dig[j] = (uint32_t)(h[j] >> shift) & 0xFFu;
}

__global__ void k_hash_place(const unsigned long long* h, const uint32_t* pos, const uint32_t* dest, uint64_t m,
                             unsigned long long* ho, uint32_t* po) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t d = dest[j];
    ho[d] = h[j];
    po[d] = pos[j];
}

void layout_hash_sort(Carve& c, HashSortLayout& L, uint64_t m) {
    const uint64_t M = m ? m : 1;
    L.dig = c.take<uint32_t>(M);
    L.dest = c.take<uint32_t>(M);
    L.h = c.take<unsigned long long>(M);
    L.pos = c.take<uint32_t>(M);
    L.ms = c.take<unsigned char>(multisplit_scratch_bytes(M, 256));
}

int hash_sort(const HashSortLayout& L, const unsigned long long* hval, const uint32_t* hpos, uint64_t m,
              unsigned long long* out_hval, uint32_t* out_hpos, cudaStream_t st) {
    if (m == 0) return DSSS_OK;
    // passes alternate between the output and L's buffers; eight passes end
    // in the output
    const unsigned long long* src_h = hval;
    const uint32_t* src_p = hpos;
    for (int pass = 0; pass < 8; ++pass) {
        unsigned long long* dh = (pass & 1) ? out_hval : L.h;
        uint32_t* dp = (pass & 1) ? out_hpos : L.pos;
        DSSS_LAUNCH("k_hash_byte", st, k_hash_byte<<<grid_for(m, 256), 256, 0, st>>>(src_h, m, 8 * pass, L.dig));
        DSSS_TRY(multisplit(L.dig, m, 256, L.dest, L.ms, st));
        DSSS_LAUNCH("k_hash_place", st,
                    k_hash_place<<<grid_for(m, 256), 256, 0, st>>>(src_h, src_p, L.dest, m, dh, dp));
        src_h = dh;
        src_p = dp;
    }
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

void layout_hash_route(Carve& c, HashRouteLayout& L, uint64_t m, uint32_t nowner) {
    const uint64_t M = m ? m : 1;
    L.owner = c.take<uint32_t>(M);
    L.dest = c.take<uint32_t>(M);
    L.counts = c.take<unsigned long long>(nowner);
    L.ms = c.take<unsigned char>(multisplit_scratch_bytes(M, nowner));
}

int hash_route(const HashRouteLayout& L, const unsigned long long* hval, const uint32_t* hpos, uint64_t m,
               uint32_t nowner, unsigned long long* out_hval, uint32_t* out_hpos, uint64_t* counts_host,
               cudaStream_t st) {
    DSSS_CUDA(cudaMemsetAsync(L.counts, 0, nowner * sizeof(unsigned long long), st));
    if (m) {
        const unsigned g = (unsigned)std::min<uint64_t>(grid_for(m, 256), 148 * 8);
        DSSS_LAUNCH("k_hash_owner", st,
                    k_hash_owner<<<g, 256, nowner * sizeof(uint32_t), st>>>(hval, m, nowner, L.owner, L.counts));
        DSSS_TRY(multisplit(L.owner, m, nowner, L.dest, L.ms, st));
        DSSS_LAUNCH("k_route_scatter", st,
                    k_route_scatter<<<grid_for(m, 256), 256, 0, st>>>(hval, hpos, L.dest, m, out_hval, out_hpos));
    }
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(counts_host, L.counts, nowner * 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

__global__ void k_dup_insert(const unsigned long long* hval, uint64_t m, unsigned long long* tkeys, uint8_t* tdup,
                             uint32_t mask, uint32_t* slot, uint32_t* err) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const unsigned long long h = hval[j];
    uint32_t sl = (uint32_t)(h ^ (h >> 32)) & mask;
    for (uint32_t probe = 0;; ++probe) {
        if (probe > mask) {
            atomicExch(err, 1u);
            sl = NO_SLOT;
            break;
        }
        const unsigned long long prev = atomicCAS(&tkeys[sl], EMPTY_KEY, h);
        if (prev == EMPTY_KEY) break;
        if (prev == h) {
            tdup[sl] = 1;
            break;
        }
        sl = (sl + 1) & mask;
    }
    slot[j] = sl;
}

__global__ void k_dup_query(const uint32_t* slot, const uint8_t* tdup, uint64_t m, uint8_t* dup) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint32_t sl = slot[j];
    dup[j] = (sl != NO_SLOT && tdup[sl]) ? 1 : 0;
}

void layout_hash_dups(Carve& c, HashDupLayout& L, uint64_t m) {
    const uint64_t M = m ? m : 1;
    L.slots = table_slots(M);
    L.tkeys = c.take<unsigned long long>(L.slots);
    L.tdup = c.take<uint8_t>(L.slots);
    L.slot = c.take<uint32_t>(M);
    L.err = c.take<uint32_t>(1);
}

int hash_dups(const HashDupLayout& L, const unsigned long long* hval, uint64_t m, uint8_t* dup, uint32_t* pin,
              cudaStream_t st) {
    if (m == 0) return DSSS_OK;
    const uint64_t slots = table_slots(m);
    DSSS_CUDA(cudaMemsetAsync(L.tkeys, 0xFF, slots * sizeof(unsigned long long), st));
    DSSS_CUDA(cudaMemsetAsync(L.tdup, 0, slots, st));
    DSSS_CUDA(cudaMemsetAsync(L.err, 0, 4, st));
    DSSS_LAUNCH("k_dup_insert", st,
                k_dup_insert<<<grid_for(m, 256), 256, 0, st>>>(hval, m, L.tkeys, L.tdup, (uint32_t)(slots - 1), L.slot,
                                                              L.err));
    DSSS_LAUNCH("k_dup_query", st, k_dup_query<<<grid_for(m, 256), 256, 0, st>>>(L.slot, L.tdup, m, dup));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(pin, L.err, 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) return fail(DSSS_EDEVICE, "duplicate test: hash table overflow");
    return DSSS_OK;
}

__global__ void k_dp_apply(const uint32_t* hpos, const uint8_t* dup, uint64_t m, uint64_t n, uint8_t* state,
                           uint32_t* err) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m || !dup[j]) return;
    const uint32_t i = hpos[j];
    if (i >= n) {
        atomicExch(err, 1u);
        return;
    }
    state[i] = 1;
}

__global__ void k_count_state(const uint8_t* state, uint64_t n, uint32_t* counters) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    block_count(counters, i < n && state[i]);
}

int dp_apply(uint32_t* counters, const uint32_t* hpos, const uint8_t* dup, uint64_t m, uint8_t* state, uint64_t n,
             uint64_t* candidates, uint32_t* pin, cudaStream_t st) {
    DSSS_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st));
    if (m) DSSS_LAUNCH("k_dp_apply", st, k_dp_apply<<<grid_for(m, 256), 256, 0, st>>>(hpos, dup, m, n, state, counters + 1));
    if (n) DSSS_LAUNCH("k_count_state", st, k_count_state<<<grid_for(n, 256), 256, 0, st>>>(state, n, counters));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaMemcpyAsync(pin, counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[1]) return fail(DSSS_EINVAL, "hash positions must be below n");
    *candidates = pin[0];
    return DSSS_OK;
}

}  // namespace dsss
