// The fused prefix-doubling path on one GPU (api.cu), for callers inside the
// library (the request server).
#pragma once
#include "internal.cuh"

namespace dsss {

// Device scratch bytes pd_sort_dev carves for n strings in nsets sets of p PEs.
uint64_t pd_scratch_bytes(uint64_t n, uint32_t nsets, uint32_t p, const dsss_opts* opts);

// dsss_pd_sort_batched on device arrays, stream st, scratch from ctx.
int pd_sort_dev(Ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p, const uint64_t* pb,
                const dsss_opts* opts, dsss_pd_result* out, cudaStream_t st);

}  // namespace dsss
