// Adjacent LCP (K4) and stable multisplit; see util.cu.
#pragma once
#include "internal.cuh"

namespace dsss {

constexpr uint32_t MAX_SPLIT_BUCKETS = 1024;

// lcp[i] = LCP(string order[i-1], string order[i]), lcp[0] = 0.
// longq: scratch of m u32, nlong: one device u32.
int adjacent_lcp(const ArenaDev& a, const uint32_t* order, uint64_t m, uint32_t* lcp, uint32_t* longq,
                 uint32_t* nlong, cudaStream_t st);

uint64_t multisplit_scratch_bytes(uint64_t n, uint32_t P);
// Stable partition by bucket id carrying up to 3 u32 columns: out[k][dest(i)]
// = in[k][i] (in[k] == NULL carries i itself); rank_out[i] (optional) = the
// position of i inside its bucket.  err: device flag set if a guard trips.
int multisplit_payload(const uint32_t* bucket, uint64_t n, uint32_t P, int npay, const uint32_t* const* in,
                       uint32_t* const* out, uint32_t* rank_out, uint32_t* err, void* scratch, cudaStream_t st);

// Stable partition by bucket id: dest[i] = output position of element i.
int multisplit(const uint32_t* bucket, uint64_t n, uint32_t P, uint32_t* dest, void* scratch, cudaStream_t st);

}  // namespace dsss
