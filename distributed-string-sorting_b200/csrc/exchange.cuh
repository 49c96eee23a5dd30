// On-device bucket scatter (K6); see exchange.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

struct ExchangeLayout {
    uint32_t* cnt;
    uint32_t* cstart;
    uint32_t* src;
    uint32_t* longq;
    uint32_t* counters;
    unsigned long long* total64;
    uint64_t* pb;
    uint64_t* bounds;
    uint64_t* slot_base;
    unsigned char* scan;
};

void layout_exchange(Carve& c, ExchangeLayout& L, uint64_t n, uint32_t p);

// Receive containers of all p PEs back to back.  recv_chars == NULL: sizes
// only (*char_total, recv_char_begin, recv_counts/offsets and the per-string
// lcp/index/pe arrays are still written).  pin: >= 8 pinned u32.
int bucket_scatter(const ExchangeLayout& L, const ArenaDev& a, uint32_t p, const uint64_t* pb,
                   const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, const uint64_t* intervals,
                   uint64_t* char_total, uint8_t* recv_chars, uint64_t recv_capacity, uint64_t* recv_char_begin,
                   uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe, uint64_t* recv_counts,
                   uint64_t* recv_offsets, uint32_t* pin, cudaStream_t st);

}  // namespace dsss
