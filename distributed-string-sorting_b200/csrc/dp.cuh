// Distinguishing-prefix rounds (K1/K2); see dp.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

struct DpLayout {
    uint8_t* st[2];
    uint8_t* kind;
    uint32_t* lens;
    uint64_t* soff;
    uint32_t* minlen;  // the shortest string of the arena (one word)
    uint32_t* slot;
    unsigned long long* tkeys;
    uint8_t* tdup;
    uint64_t slots;
    uint32_t* counters;
    // independent string sets (batched sorts): sorted positions
    // [set_begin[s], set_begin[s+1]) belong to set s; each set hashes into its
    // own region [set_base[s], set_base[s] + set_mask[s] + 1) of the table
    uint32_t nsets_cap;
    uint64_t* set_begin;
    uint64_t* set_base;
    uint32_t* set_mask;
    uint32_t* set_cnt;
    // fingerprint filter (planned when n >= filter_min): bitmap words,
    // per-position hashes, candidate positions, per-set filter regions
    uint64_t filter_min;
    uint32_t filter_bpk;
    uint64_t bm_words;
    uint32_t* bits;
    unsigned long long* hbuf;  // also the stored hashes of the split hash round
    uint32_t* cand;
    bool split;  // hash round as k_dp_hash_store + k_dp_insert
    // dense rounds (hashed * digest_share >= positions) in arena order: the
    // hashed strings (hmask), the strings whose hash is shared (dmask), both
    // bitmaps over arena indices, and the first inserting string of every
    // table slot (tid)
    uint32_t digest_share;
    uint32_t* hmask;
    uint32_t* dmask;
    uint64_t mask_words;
    uint32_t* tid;
    // dense rounds without the table: (hash, string) pairs partitioned by
    // the hash's top bits in two radix passes into at most pd_nb buckets,
    // each deduplicated in shared memory: the pairs after the first pass
    // (pp_h1 / pp_s1) and after the second (pd_h / pd_s), the buckets' starts
    // (pd_start, pd_nb + 1), the round's hashes in arena order when the sort
    // did not store them (pp_dig), per-tile counts and their scan (pp_hist,
    // pp_off: pp_hcap and 2 pp_hcap entries), the coarse buckets' layout
    // (pp_mid) and the passes' totals (pp_total)
    uint32_t pd_nb;
    uint32_t* pd_start;
    unsigned long long* pd_h;
    uint32_t* pd_s;
    unsigned long long* pp_h1;
    uint32_t* pp_s1;
    unsigned long long* pp_dig;
    uint32_t* pp_hist;
    uint32_t* pp_off;
    uint64_t pp_hcap;
    uint32_t* pp_mid;
    uint32_t* pp_total;
    unsigned char* pp_scan;
    uint64_t* set_bbase;
    uint32_t* set_bmask;
    uint32_t* set_ccnt;
};

void layout_dp(Carve& c, DpLayout& L, uint64_t n, uint32_t nsets = 1);

// order/lcp: strings in sorted order per PE (lcp 0 at every PE start); dp[i]
// receives the distinguishing-prefix length of the string at position i.
// set_begin_host (nsets + 1 bounds, NULL for one set): prefixes are only
// duplicates of prefixes in the same set.
// rdig (optional): the string sort's prefix hashes at the first schedule
// depths (ROOT_DIGESTS arrays of a.n entries, array j for depth
// root_digest_depth(j), valid where bit j of rdig_mask is set), read by the
// arena-order rounds at those depths.
int dp_rounds(const DpLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
              uint32_t* dp, uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds, uint32_t* pin,
              cudaStream_t st, uint32_t nsets = 1, const uint64_t* set_begin_host = nullptr,
              const unsigned long long* rdig = nullptr, uint32_t rdig_mask = 0);

struct DpRoundLayout {
    DpLayout dp;
    uint32_t* flag;
    uint32_t* pos;
    uint32_t* total;
    unsigned char* scan;
};

void layout_dp_round(Carve& c, DpRoundLayout& R, uint64_t n);

// One BloomFilter::filter round: cand (ascending sorted positions, or NULL for
// every position, the first round) at depth; dp[c] written for each
// candidate; next receives the surviving positions, *m_next their count.
int dp_one_round(const DpRoundLayout& R, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
                 const uint32_t* cand, uint64_t m, uint32_t depth, uint32_t* dp, uint32_t* next, uint64_t* m_next,
                 uint32_t* pin, cudaStream_t st);

int prefix_hash(const ArenaDev& a, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* out,
                cudaStream_t st);

// ---- PEs on several GPUs: one round split around the hash exchange ----
struct DpSplitLayout {
    uint32_t* lens;
    uint64_t* soff;
    uint8_t* kind;
    uint32_t* flag;
    uint32_t* pos;
    uint32_t* counters;
    unsigned char* scan;
};
void layout_dp_split(Carve& c, DpSplitLayout& L, uint64_t n);

// Classifies the round at depth (state_in NULL: every position is a
// candidate); dp gets the depth (or the length) of every candidate,
// state_out the LCP duplicates and roots, and (hpos, hval)[0..*m) the
// positions and hashes of every hashed candidate, in position order.
int dp_classify_hash(const DpSplitLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
                     const uint8_t* state_in, uint32_t depth, uint32_t* dp, uint8_t* state_out, uint32_t* hpos,
                     unsigned long long* hval, uint64_t* m, uint32_t* pin, cudaStream_t st);

struct HashRouteLayout {
    uint32_t* owner;
    uint32_t* dest;
    unsigned long long* counts;
    void* ms;
};
void layout_hash_route(Carve& c, HashRouteLayout& L, uint64_t m, uint32_t nowner);

// Groups (hval, hpos) by owner GPU (equal slices of the hash range), stable;
// counts_host[nowner] the group sizes.
int hash_route(const HashRouteLayout& L, const unsigned long long* hval, const uint32_t* hpos, uint64_t m,
               uint32_t nowner, unsigned long long* out_hval, uint32_t* out_hpos, uint64_t* counts_host,
               cudaStream_t st);

struct HashSortLayout {
    uint32_t* dig;
    uint32_t* dest;
    unsigned long long* h;
    uint32_t* pos;
    void* ms;
};
void layout_hash_sort(Carve& c, HashSortLayout& L, uint64_t m);

// (hval, hpos) in ascending hash order, stable (out may not alias in).
int hash_sort(const HashSortLayout& L, const unsigned long long* hval, const uint32_t* hpos, uint64_t m,
              unsigned long long* out_hval, uint32_t* out_hpos, cudaStream_t st);

struct HashDupLayout {
    uint64_t slots;
    unsigned long long* tkeys;
    uint8_t* tdup;
    uint32_t* slot;
    uint32_t* err;
};
void layout_hash_dups(Carve& c, HashDupLayout& L, uint64_t m);

// dup[j] = 1 iff hval[j] occurs at least twice in hval[0..m).
int hash_dups(const HashDupLayout& L, const unsigned long long* hval, uint64_t m, uint8_t* dup, uint32_t* pin,
              cudaStream_t st);

// state[hpos[j]] = 1 where dup[j]; *candidates = the positions with state 1.
// counters: 2 device u32.
int dp_apply(uint32_t* counters, const uint32_t* hpos, const uint8_t* dup, uint64_t m, uint8_t* state, uint64_t n,
             uint64_t* candidates, uint32_t* pin, cudaStream_t st);

}  // namespace dsss
