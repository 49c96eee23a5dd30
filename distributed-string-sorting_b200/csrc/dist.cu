// C ABI entries for PEs spread over several GPUs (one process per GPU): the
// pieces of the prefix-doubling path around its three exchanges, which the
// caller carries out with its collective library (NCCL through
// torch.distributed in distributed-string-sorting_b200/dist.py):
//   1. every distinguishing-prefix round: hashes of this GPU's candidates,
//      routed to the GPU owning their slice of the hash range, tested there
//      for duplicates, the outcome sent back and applied;
//   2. the splitter sample: each GPU packs its samples, all GPUs sort the
//      gathered sample and search their PEs for the splitters;
//   3. the string exchange: each GPU packs one receive container per
//      destination PE, the containers travel, and the receiving GPU regroups
//      them by receiver before the LCP merge (dsss_lcp_merge).
#include <algorithm>
#include <vector>

#include "dp.cuh"
#include "exchange.cuh"
#include "internal.cuh"
#include "partition.cuh"
#include "util.cuh"

namespace dsss {

static ArenaDev view(const dsss_arena* a) { return ArenaDev{a->chars, a->offsets, a->lengths, a->n}; }

// ------------------------------------------------------------------ pack ----
__global__ void k_pack_sizes(ArenaDev a, const uint32_t* ids, const uint32_t* trunc, uint64_t m, uint32_t* size,
                             uint32_t* plen) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    uint64_t off;
    uint32_t len;
    str_of(a, ids[j], off, len);
    if (trunc) len = min(len, trunc[j]);
    plen[j] = len;
    size[j] = len + 1;
}

__global__ void k_pack_copy(ArenaDev a, const uint32_t* ids, const uint32_t* plen, const uint64_t* out_off, uint64_t m,
                            uint8_t* out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    uint64_t off;
    uint32_t len;
    str_of(a, ids[j], off, len);
    const uint32_t l = plen[j];
    const uint8_t* src = a.chars + off;
    uint8_t* dst = out + out_off[j];
    for (uint32_t k = 0; k < l; ++k) dst[k] = src[k];
    dst[l] = 0;
}

// --------------------------------------------------------------- regroup ----
// Block table entry: (src string, dst string, strings, src byte, dst byte, bytes).
__global__ void k_regroup_starts(const uint64_t* blk, uint32_t nblk, const uint64_t* dst_first, uint64_t n,
                                 const uint32_t* src_start, uint32_t* dst_start) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t lo = 0, hi = nblk;  // block of destination string i: last b with dst_first[b] <= i
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (dst_first[mid] <= i) lo = mid;
        else hi = mid;
    }
    const uint64_t* b = blk + 6 * (uint64_t)lo;
    const uint64_t k = i - b[1];
    dst_start[i] = (uint32_t)(src_start[b[0] + k] + b[4]);
}

}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_dp_classify_hash(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, const uint32_t* lcp,
                          const uint8_t* state_in, uint32_t depth, uint32_t* dp, uint8_t* state_out, uint32_t* hpos,
                          uint64_t* hval, uint64_t* m, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    if (!m) return fail(DSSS_EINVAL, "m is NULL");
    if (in->n && (!order || !lcp || !dp || !state_out || !hpos || !hval))
        return fail(DSSS_EINVAL, "order/lcp/dp/state_out/hpos/hval is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    DpSplitLayout L;
    layout_dp_split(sz, L, in->n);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_dp_split(c, L, in->n);
    return dp_classify_hash(L, view(in), in->n, order, lcp, state_in, depth, dp, state_out, hpos,
                            (unsigned long long*)hval, m, (uint32_t*)ctx->pin, (cudaStream_t)stream);
}

int dsss_hash_route(dsss_ctx* ctx, const uint64_t* hval, const uint32_t* hpos, uint64_t m, uint32_t nowner,
                    uint64_t* out_hval, uint32_t* out_hpos, uint64_t* counts, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (nowner == 0 || nowner > MAX_SPLIT_BUCKETS)
        return fail(DSSS_EINVAL, "nowner must be in 1..%u", MAX_SPLIT_BUCKETS);
    if (!counts || (m && (!hval || !hpos || !out_hval || !out_hpos))) return fail(DSSS_EINVAL, "array is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    HashRouteLayout L;
    layout_hash_route(sz, L, m, nowner);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    Carve c(ctx->ws);
    layout_hash_route(c, L, m, nowner);
    return hash_route(L, (const unsigned long long*)hval, hpos, m, nowner, (unsigned long long*)out_hval, out_hpos,
                      counts, (cudaStream_t)stream);
}

int dsss_hash_sort(dsss_ctx* ctx, const uint64_t* hval, const uint32_t* hpos, uint64_t m, uint64_t* out_hval,
                   uint32_t* out_hpos, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (m && (!hval || !hpos || !out_hval || !out_hpos)) return fail(DSSS_EINVAL, "array is NULL");
    if (m && ((const void*)hval == (const void*)out_hval || (const void*)hpos == (const void*)out_hpos))
        return fail(DSSS_EINVAL, "the output may not be the input");
    if (m >= (1ull << 32)) return fail(DSSS_ENOTSUP, "2^32 or more hash records");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    HashSortLayout L;
    layout_hash_sort(sz, L, m);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    Carve c(ctx->ws);
    layout_hash_sort(c, L, m);
    return hash_sort(L, (const unsigned long long*)hval, hpos, m, (unsigned long long*)out_hval, out_hpos,
                     (cudaStream_t)stream);
}

int dsss_hash_dups(dsss_ctx* ctx, const uint64_t* hval, uint64_t m, uint8_t* dup, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (m && (!hval || !dup)) return fail(DSSS_EINVAL, "hval/dup is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    HashDupLayout L;
    layout_hash_dups(sz, L, m);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_hash_dups(c, L, m);
    return hash_dups(L, (const unsigned long long*)hval, m, dup, (uint32_t*)ctx->pin, (cudaStream_t)stream);
}

int dsss_dp_apply(dsss_ctx* ctx, const uint32_t* hpos, const uint8_t* dup, uint64_t m, uint8_t* state, uint64_t n,
                  uint64_t* candidates, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (!candidates || (m && (!hpos || !dup)) || (n && !state)) return fail(DSSS_EINVAL, "array is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    DSSS_TRY(ensure_ws(ctx, 256));
    DSSS_TRY(ensure_pin(ctx, 4096));
    return dp_apply((uint32_t*)ctx->ws, hpos, dup, m, state, n, candidates, (uint32_t*)ctx->pin,
                    (cudaStream_t)stream);
}

int dsss_pack_strings(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* ids, const uint32_t* trunc, uint64_t m,
                      uint8_t* out_chars, uint64_t capacity, uint64_t* out_offsets, uint32_t* out_lengths,
                      uint64_t* bytes, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    if (!bytes || (m && (!ids || !out_offsets || !out_lengths))) return fail(DSSS_EINVAL, "array is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    *bytes = 0;
    if (m == 0) return DSSS_OK;
    Carve sz(nullptr);
    sz.take<uint32_t>(m);
    sz.take<uint64_t>(1);
    sz.take<unsigned char>(scan_scratch_bytes(m));
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    uint32_t* size = c.take<uint32_t>(m);
    uint64_t* total = c.take<uint64_t>(1);
    void* scan = c.take<unsigned char>(scan_scratch_bytes(m));
    const ArenaDev a = view(in);
    DSSS_LAUNCH("k_pack_sizes", st, k_pack_sizes<<<grid_for(m, 256), 256, 0, st>>>(a, ids, trunc, m, size, out_lengths));
    DSSS_TRY(exclusive_scan_u32_to_u64(size, out_offsets, m, total, scan, st));
    DSSS_CUDA(cudaMemcpyAsync(ctx->pin, total, 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    *bytes = *(const uint64_t*)ctx->pin;
    if (!out_chars) return DSSS_OK;
    if (capacity < *bytes)
        return fail(DSSS_EINVAL, "pack buffer of %llu bytes < %llu needed", (unsigned long long)capacity,
                    (unsigned long long)*bytes);
    DSSS_LAUNCH("k_pack_copy", st,
                k_pack_copy<<<grid_for(m, 256), 256, 0, st>>>(a, ids, out_lengths, out_offsets, m, out_chars));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

int dsss_partition_search(dsss_ctx* ctx, const dsss_arena* in, uint32_t p_local, const uint64_t* part_begin,
                          const uint32_t* local_order, const dsss_arena* splitters, const uint64_t* spl_index,
                          uint32_t p_global, const uint64_t* pe_index, int indexed, uint64_t* intervals,
                          dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    DSSS_TRY(check_arena(splitters));
    if (p_local == 0 || p_global == 0) return fail(DSSS_EINVAL, "p_local/p_global must be >= 1");
    if (!part_begin || !intervals || (in->n && !local_order)) return fail(DSSS_EINVAL, "array is NULL");
    if (part_begin[0] != 0 || part_begin[p_local] != in->n) return fail(DSSS_EINVAL, "part_begin must span 0..n");
    if (indexed && ((splitters->n && !spl_index) || !pe_index)) return fail(DSSS_EINVAL, "indices missing");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return partition_search(ctx, view(in), p_local, part_begin, local_order, view(splitters), spl_index, p_global,
                            pe_index, indexed, intervals, (cudaStream_t)stream);
}

int dsss_bucket_send(dsss_ctx* ctx, const dsss_arena* in, uint32_t p_local, const uint64_t* part_begin,
                     const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, uint32_t p_global,
                     uint32_t q_first, const uint64_t* intervals, uint8_t* send_chars, uint64_t capacity,
                     uint64_t* char_total, uint64_t* recv_char_begin, uint32_t* char_start, uint32_t* send_lcp,
                     uint64_t* counts, uint64_t* offsets, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    if (p_local == 0 || p_global == 0 || q_first + p_local > p_global) return fail(DSSS_EINVAL, "bad PE counts");
    if (!part_begin || !intervals || !char_total) return fail(DSSS_EINVAL, "array is NULL");
    if (part_begin[0] != 0 || part_begin[p_local] != in->n) return fail(DSSS_EINVAL, "part_begin must span 0..n");
    if (in->n && (!local_order || !lcp || !dp || !send_lcp)) return fail(DSSS_EINVAL, "array is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    ExchangeLayout L;
    layout_exchange(sz, L, in->n, p_local, p_global);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_exchange(c, L, in->n, p_local, p_global);
    cudaStream_t st = (cudaStream_t)stream;
    DSSS_TRY(bucket_scatter_rect(L, view(in), p_local, p_global, q_first, part_begin, local_order, lcp, dp, intervals,
                                 char_total, send_chars, capacity, recv_char_begin, char_start, true, send_lcp, nullptr,
                                 nullptr, counts, offsets, (uint32_t*)ctx->pin, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

int dsss_regroup(dsss_ctx* ctx, uint32_t nblocks, const uint64_t* blocks, const uint8_t* src_chars,
                 uint8_t* dst_chars, const uint32_t* src_start, uint32_t* dst_start, const uint32_t* src_lcp,
                 uint32_t* dst_lcp, uint64_t n, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (nblocks && !blocks) return fail(DSSS_EINVAL, "blocks is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    // the blocks must tile the destination strings in order
    std::vector<uint64_t> first(nblocks + 1);
    uint64_t next = 0;
    for (uint32_t b = 0; b < nblocks; ++b) {
        const uint64_t* e = blocks + 6 * (uint64_t)b;
        if (e[1] != next) return fail(DSSS_EINVAL, "block %u does not start where the previous one ends", b);
        first[b] = e[1];
        next = e[1] + e[2];
    }
    if (next != n)
        return fail(DSSS_EINVAL, "blocks cover %llu strings, not %llu", (unsigned long long)next,
                    (unsigned long long)n);
    first[nblocks] = n;
    for (uint32_t b = 0; b < nblocks; ++b) {
        const uint64_t* e = blocks + 6 * (uint64_t)b;
        if (e[5]) DSSS_CUDA(cudaMemcpyAsync(dst_chars + e[4], src_chars + e[3], e[5], cudaMemcpyDeviceToDevice, st));
        if (e[2]) DSSS_CUDA(cudaMemcpyAsync(dst_lcp + e[1], src_lcp + e[0], e[2] * 4, cudaMemcpyDeviceToDevice, st));
    }
    if (n) {
        Carve sz(nullptr);
        sz.take<uint64_t>(6ull * nblocks + 1);
        sz.take<uint64_t>(nblocks + 1);
        DSSS_TRY(ensure_ws(ctx, sz.used));
        Carve c(ctx->ws);
        uint64_t* d_blk = c.take<uint64_t>(6ull * nblocks + 1);
        uint64_t* d_first = c.take<uint64_t>(nblocks + 1);
        DSSS_CUDA(cudaMemcpyAsync(d_blk, blocks, 6ull * nblocks * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(d_first, first.data(), (nblocks + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_regroup_starts", st,
                    k_regroup_starts<<<grid_for(n, 256), 256, 0, st>>>(d_blk, nblocks, d_first, n, src_start,
                                                                      dst_start));
    }
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

}  // extern "C"
