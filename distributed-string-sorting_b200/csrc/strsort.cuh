// Segmented MSD string sort with LCP output (K3); see strsort.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

struct SortLayout {
    uint32_t* ord[2];
    unsigned long long* key[2];
    unsigned char* large[2];
    unsigned char* small[4];
    uint32_t* tile0;
    uint32_t* chunk0;
    uint32_t* tmp_counts;
    uint32_t* tile_hist;
    uint32_t* chunk_pre;
    uint32_t* bucket;
    uint32_t* child;  // 256 per large segment (NULL: the passes read the keys themselves)
    uint32_t* counters;
    uint64_t* pb;
    unsigned char* scan;
    unsigned long long* spl;  // sampled splitter tables
    uint32_t* fix;            // bucket starts whose LCP is written at the end
    uint32_t* pin;
    uint64_t cap_large, cap_small, cap_tiles, cap_chunks, cap_spl, cap_fix;
};

constexpr uint32_t SORT_SMALL_MAX_DEFAULT = 4096;

// Scratch layout for sorting up to n strings in up to p segments.
void layout_sort(Carve& c, SortLayout& L, uint64_t n, uint32_t p, uint32_t small_max);

// Sorts ids (ids_in[i], or i when ids_in is NULL) within the segments
// [pb[q], pb[q+1]) by the bytes of their strings.  ord_out gets the sorted ids,
// lcp_out[i] the LCP with position i-1 (0 at segment starts).  pin: pinned
// host buffer of >= 16 u32 for count read-backs (the call synchronises on st).
// dig (optional, ROOT_DIGESTS * n entries): the first pass stores every
// string's prefix hashes at the first schedule depths there (root_digests,
// array j at dig + j * n); bit j of *dig_mask tells whether array j holds
// every string's hash (the ids are the arena's, every string went through
// that pass and no segment skipped depth j).
// seg_depth (optional, device, p entries): the strings of segment q share
// their first seg_depth[q] bytes (the sort starts there).
int sort_strings(const SortLayout& L, const ArenaDev& a, uint64_t n, uint32_t p, const uint64_t* pb_host,
                 const uint32_t* ids_in, uint32_t* ord_out, uint32_t* lcp_out, uint32_t small_max,
                 uint32_t* pin, cudaStream_t st, unsigned long long* dig = nullptr, uint32_t* dig_mask = nullptr,
                 const uint32_t* seg_depth = nullptr);

}  // namespace dsss
