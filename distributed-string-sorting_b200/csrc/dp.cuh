// Distinguishing-prefix rounds (K1/K2); see dp.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

struct DpLayout {
    uint8_t* st[2];
    uint8_t* kind;
    uint32_t* lens;
    uint64_t* soff;
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
    unsigned long long* hbuf;
    uint32_t* cand;
    uint64_t* set_bbase;
    uint32_t* set_bmask;
    uint32_t* set_ccnt;
};

void layout_dp(Carve& c, DpLayout& L, uint64_t n, uint32_t nsets = 1);

// order/lcp: strings in sorted order per PE (lcp 0 at every PE start); dp[i]
// receives the distinguishing-prefix length of the string at position i.
// set_begin_host (nsets + 1 bounds, NULL for one set): prefixes are only
// duplicates of prefixes in the same set.
int dp_rounds(const DpLayout& L, const ArenaDev& a, uint64_t n, const uint32_t* order, const uint32_t* lcp,
              uint32_t* dp, uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds, uint32_t* pin,
              cudaStream_t st, uint32_t nsets = 1, const uint64_t* set_begin_host = nullptr);

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

}  // namespace dsss
