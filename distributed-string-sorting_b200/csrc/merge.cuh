// Merge of prefix-compressed receive containers (K7); see merge.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

struct MergeJob;

struct MergeLayout {
    uint32_t* start;
    uint32_t* flag;
    uint32_t* pos;
    uint32_t* flen;
    uint64_t* foff;
    uint32_t* tree;
    uint8_t* full;
    uint32_t* ids[2];
    uint32_t* l[2];
    uint8_t* run_start;
    uint32_t* run_of;
    uint32_t* run_begin;
    uint32_t* run_len;
    uint64_t* run_offset;
    MergeJob* jobs;
    uint32_t* counters;
    uint64_t* total64;
    unsigned char* scan;
};

void layout_merge(Carve& c, MergeLayout& L, uint64_t n, uint64_t bytes, uint64_t full_bytes, uint32_t nruns);

// nrecv receive containers back to back, each of p source runs
// (counts/offsets: host, nrecv*p, [r*p + q]).  Outputs per merged position:
// order (index into the containers), merged_lcp, old_lcp (the sender-side LCP,
// 0 at run starts), perm_index/perm_pe (sender local index and sender PE);
// any output may be NULL except order.
int lcp_merge(Ctx* ctx, const uint8_t* chars, uint64_t bytes, const uint32_t* char_start, const uint32_t* lcp,
              uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* counts, const uint64_t* offsets,
              uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp, uint32_t* perm_index, uint32_t* perm_pe,
              cudaStream_t st);

// lcp_merge, then every merged string whole (prefixes decompressed),
// NUL-terminated, back to back in merged order: out_offsets/out_lengths per
// merged position, *out_bytes the bytes written (or needed: DSSS_EINVAL when
// out_capacity is below them).
int lcp_merge_strings(Ctx* ctx, const uint8_t* chars, uint64_t bytes, const uint32_t* char_start, const uint32_t* lcp,
                      uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* counts, const uint64_t* offsets,
                      uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp, uint32_t* perm_index,
                      uint32_t* perm_pe, uint8_t* out_chars, uint64_t out_capacity, uint64_t* out_offsets,
                      uint32_t* out_lengths, uint64_t* out_bytes, cudaStream_t st);

}  // namespace dsss
