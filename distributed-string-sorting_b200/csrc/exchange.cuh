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
    uint64_t* rbeg;
    unsigned char* scan;
};

// Scratch for ps sending and pr receiving PEs (pr = 0: pr = ps).
void layout_exchange(Carve& c, ExchangeLayout& L, uint64_t n, uint32_t ps, uint32_t pr = 0);

// Receive containers of all p PEs back to back.  recv_chars == NULL: sizes
// only (*char_total, recv_char_begin, recv_counts/offsets and the per-string
// lcp/index/pe arrays are still written).  pin: >= 8 pinned u32.
int bucket_scatter(const ExchangeLayout& L, const ArenaDev& a, uint32_t p, const uint64_t* pb,
                   const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, const uint64_t* intervals,
                   uint64_t* char_total, uint8_t* recv_chars, uint64_t recv_capacity, uint64_t* recv_char_begin,
                   uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe, uint64_t* recv_counts,
                   uint64_t* recv_offsets, uint32_t* pin, cudaStream_t st);

// The same with ps sending PEs (global ids q_first..) and pr receiving PEs:
// the containers of all pr receivers back to back, each holding the
// intervals[q*pr + r] strings of every sender q; recv_counts/recv_offsets
// [r*ps + q].  recv_char_start (optional): each string's first byte, relative
// to its receiver's container if starts_per_receiver, else to recv_chars.
int bucket_scatter_rect(const ExchangeLayout& L, const ArenaDev& a, uint32_t ps, uint32_t pr, uint32_t q_first,
                        const uint64_t* pb, const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp,
                        const uint64_t* intervals, uint64_t* char_total, uint8_t* recv_chars, uint64_t recv_capacity,
                        uint64_t* recv_char_begin, uint32_t* recv_char_start, bool starts_per_receiver,
                        uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe, uint64_t* recv_counts,
                        uint64_t* recv_offsets, uint32_t* pin, cudaStream_t st);

}  // namespace dsss
