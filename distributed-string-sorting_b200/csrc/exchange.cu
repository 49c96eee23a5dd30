// K6 — on-device bucket scatter: AllToAllStringImplPrefixDoubling::alltoallv
// (src/mpi/alltoall.hpp:910-1008) with EmptyPrefixDoublingLcpByteEncoderMemCpy
// (src/mpi/byte_encoder.hpp:139-171) for p PEs that share one GPU.
//
// PE r's receive container holds, in source-PE order, the r-th interval of
// every PE (intervals[q*p + r] strings of PE q's local order).  Each string
// contributes bytes [lcp', dp) and a NUL, where lcp' is its local LCP except
// 0 at the first string of every non-empty interval (setLcpAtStartOfInterval,
// alltoall.hpp:396-404); its tag is (index in the sender's local order,
// sender PE) (InitPolicy<IndexPEIndex>, strings/stringcontainer.hpp:127-158).
//
// One thread per string computes its receive slot arithmetically (no sort:
// slots follow from the interval table), a scan turns byte counts into
// offsets, and a copy kernel gathers the bytes — warp-cooperative for long
// strings.
#include <vector>

#include "exchange.cuh"
#include "internal.cuh"

namespace dsss {

// ps sending PEs (this call's strings) and pr receiving PEs; the senders'
// global PE ids start at q_first.
__global__ void k_recv_slots(ArenaDev a, const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp,
                             const uint64_t* pb, const uint64_t* bounds, const uint64_t* slot_base, uint32_t ps,
                             uint32_t pr, uint32_t q_first, uint64_t n, uint32_t* cnt, uint32_t* rlcp,
                             uint32_t* rindex, uint32_t* rpe, uint32_t* rsrc, uint32_t* err) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    uint32_t lo = 0, hi = ps;  // PE of local position g: last q with pb[q] <= g
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (pb[mid] <= g) lo = mid;
        else hi = mid;
    }
    const uint32_t q = lo;
    const uint64_t i = g - pb[q];
    const uint64_t* b = bounds + (uint64_t)q * (pr + 1);
    lo = 0;
    hi = pr;  // bucket: last r with b[r] <= i
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (b[mid] <= i) lo = mid;
        else hi = mid;
    }
    const uint32_t r = lo;
    const uint32_t l = i == b[r] ? 0u : lcp[g];
    const uint32_t d = dp[g];
    if (d < l) {  // a DP shorter than the LCP cannot come from a consistent local sort
        atomicExch(err, 1u);
        return;
    }
    const uint64_t o = slot_base[(uint64_t)r * ps + q] + (i - b[r]);
    if (o >= n) {
        atomicExch(err, 1u);
        return;
    }
    cnt[o] = d - l + 1;
    rlcp[o] = l;
    if (rindex) rindex[o] = (uint32_t)i;
    if (rpe) rpe[o] = q_first + q;
    rsrc[o] = local_order[g];
}

// Char starts relative to each receiver's container (rbeg: pr + 1 slot bounds).
__global__ void k_rel_starts(const uint32_t* cstart, uint64_t n, const uint64_t* rbeg, uint32_t pr, uint32_t* out) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    uint32_t lo = 0, hi = pr;  // receiver of slot o: last r with rbeg[r] <= o
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (rbeg[mid] <= o) lo = mid;
        else hi = mid;
    }
    out[o] = cstart[o] - cstart[rbeg[lo]];
}

__global__ void k_sum_u32(const uint32_t* v, uint64_t n, unsigned long long* total) {
    unsigned long long s = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += v[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

// Copies bytes [lcp, lcp + cnt - 1) of each source string and a NUL.  Up to
// COPY_GROUP_MAX bytes: a group of COPY_LANES lanes per string, so that one
// warp instruction stores COPY_LANES consecutive bytes of each of 32 /
// COPY_LANES strings instead of one byte of each of 32; longer strings: one
// warp each (queued).
constexpr uint32_t COPY_LANES = 8, COPY_GROUP_MAX = 256;

__global__ void k_recv_copy(ArenaDev a, uint64_t n, const uint32_t* cnt, const uint32_t* cstart, const uint32_t* rlcp,
                            const uint32_t* rsrc, uint8_t* out, uint32_t* longq, uint32_t* nlong) {
    const uint64_t o = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / COPY_LANES;
    const uint32_t lane = threadIdx.x % COPY_LANES;
    if (o >= n) return;
    const uint32_t m = cnt[o] - 1;
    uint8_t* dst = out + cstart[o];
    if (lane == 0) dst[m] = 0;
    if (m > COPY_GROUP_MAX) {
        if (lane == 0) longq[atomicAdd(nlong, 1u)] = (uint32_t)o;
        return;
    }
    uint64_t off;
    uint32_t len;
    str_of(a, rsrc[o], off, len);
    // byte by byte: these strings are short (DP - lcp), where copy_words' head
    // and tail cost more than its whole-word stores save (6.42 vs 6.05 ms)
    const uint8_t* src = a.chars + off + rlcp[o];
#pragma unroll 4
    for (uint32_t k = lane; k < m; k += COPY_LANES) dst[k] = src[k];
}

__global__ void k_recv_copy_warp(ArenaDev a, const uint32_t* cnt, const uint32_t* cstart, const uint32_t* rlcp,
                                 const uint32_t* rsrc, uint8_t* out, const uint32_t* longq, const uint32_t* nlong) {
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t total = *nlong;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += nw) {
        const uint32_t o = longq[w];
        const uint32_t m = cnt[o] - 1;
        uint64_t off;
        uint32_t len;
        str_of(a, rsrc[o], off, len);
        const uint8_t* src = a.chars + off + rlcp[o];
        uint8_t* dst = out + cstart[o];
        for (uint32_t k = lane; k < m; k += 32) dst[k] = src[k];
    }
}

void layout_exchange(Carve& c, ExchangeLayout& L, uint64_t n, uint32_t ps, uint32_t pr) {
    if (pr == 0) pr = ps;
    uint64_t N = n ? n : 1;
    L.cnt = c.take<uint32_t>(N);
    L.cstart = c.take<uint32_t>(N);
    L.src = c.take<uint32_t>(N);
    L.longq = c.take<uint32_t>(N);
    L.counters = c.take<uint32_t>(4);
    L.total64 = c.take<unsigned long long>(1);
    L.pb = c.take<uint64_t>(ps + 1);
    L.bounds = c.take<uint64_t>((uint64_t)ps * (pr + 1));
    L.slot_base = c.take<uint64_t>((uint64_t)ps * pr);
    L.rbeg = c.take<uint64_t>(pr + 1);
    L.scan = c.take<unsigned char>(scan_scratch_bytes(N));
}

int bucket_scatter_rect(const ExchangeLayout& L, const ArenaDev& a, uint32_t ps, uint32_t pr, uint32_t q_first,
                        const uint64_t* pb, const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp,
                        const uint64_t* intervals, uint64_t* char_total, uint8_t* recv_chars, uint64_t recv_capacity,
                        uint64_t* recv_char_begin, uint32_t* recv_char_start, bool starts_per_receiver,
                        uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe, uint64_t* recv_counts,
                        uint64_t* recv_offsets, uint32_t* pin, cudaStream_t st) {
    const uint64_t n = pb[ps];
    // interval bounds per sender, receive slots per (receiver, sender)
    std::vector<uint64_t> bounds((uint64_t)ps * (pr + 1)), slot((uint64_t)pr * ps), rbeg(pr + 1, 0);
    for (uint32_t q = 0; q < ps; ++q) {
        bounds[(uint64_t)q * (pr + 1)] = 0;
        uint64_t tot = 0;
        for (uint32_t r = 0; r < pr; ++r) {
            tot += intervals[(uint64_t)q * pr + r];
            bounds[(uint64_t)q * (pr + 1) + r + 1] = tot;
        }
        if (tot != pb[q + 1] - pb[q]) return fail(DSSS_EINVAL, "intervals of PE %u do not add up to its size", q);
    }
    for (uint32_t r = 0; r < pr; ++r) {
        uint64_t run = rbeg[r];
        for (uint32_t q = 0; q < ps; ++q) {
            slot[(uint64_t)r * ps + q] = run;
            if (recv_counts) recv_counts[(uint64_t)r * ps + q] = intervals[(uint64_t)q * pr + r];
            if (recv_offsets) recv_offsets[(uint64_t)r * ps + q] = bounds[(uint64_t)q * (pr + 1) + r];
            run += intervals[(uint64_t)q * pr + r];
        }
        rbeg[r + 1] = run;
    }
    if (n == 0) {
        *char_total = 0;
        if (recv_char_begin)
            for (uint32_t r = 0; r <= pr; ++r) recv_char_begin[r] = 0;
        return DSSS_OK;
    }
    DSSS_CUDA(cudaMemsetAsync(L.counters, 0, 4 * sizeof(uint32_t), st));
    DSSS_CUDA(cudaMemcpyAsync(L.pb, pb, (ps + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.bounds, bounds.data(), bounds.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.slot_base, slot.data(), slot.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.rbeg, rbeg.data(), rbeg.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_LAUNCH("k_recv_slots", st,
                k_recv_slots<<<grid_for(n, 256), 256, 0, st>>>(a, local_order, lcp, dp, L.pb, L.bounds, L.slot_base,
                                                              ps, pr, q_first, n, L.cnt, recv_lcp, recv_index, recv_pe,
                                                              L.src, L.counters + 2));
    DSSS_TRY(exclusive_scan_u32(L.cnt, L.cstart, n, L.counters, L.scan, st));
    DSSS_CUDA(cudaMemsetAsync(L.total64, 0, 8, st));
    DSSS_LAUNCH("k_sum_u32", st, k_sum_u32<<<148 * 4, 256, 0, st>>>(L.cnt, n, L.total64));
    DSSS_CUDA(cudaMemcpyAsync(pin, L.counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(pin + 4, L.total64, 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[2]) return fail(DSSS_EINVAL, "dp shorter than lcp: order/lcp/dp are not a local sort");
    const uint64_t total64 = *(const uint64_t*)(pin + 4);
    if (total64 >= (1ull << 32)) return fail(DSSS_ENOTSUP, "receive containers over 4 GiB per call");
    *char_total = pin[0];
    if (recv_char_begin) {
        std::vector<uint32_t> cs(pr + 1);
        for (uint32_t r = 0; r < pr; ++r) {
            if (rbeg[r] < n) DSSS_CUDA(cudaMemcpyAsync(&cs[r], L.cstart + rbeg[r], 4, cudaMemcpyDeviceToHost, st));
            else cs[r] = pin[0];
        }
        DSSS_CUDA(cudaStreamSynchronize(st));
        for (uint32_t r = 0; r < pr; ++r) recv_char_begin[r] = cs[r];
        recv_char_begin[pr] = pin[0];
    }
    if (recv_char_start) {
        if (starts_per_receiver)
            DSSS_LAUNCH("k_rel_starts", st,
                        k_rel_starts<<<grid_for(n, 256), 256, 0, st>>>(L.cstart, n, L.rbeg, pr, recv_char_start));
        else
            DSSS_CUDA(cudaMemcpyAsync(recv_char_start, L.cstart, n * 4, cudaMemcpyDeviceToDevice, st));
    }
    if (!recv_chars) return DSSS_OK;
    if (recv_capacity < *char_total) return fail(DSSS_EINVAL, "receive buffer of %llu bytes < %llu needed",
                                                 (unsigned long long)recv_capacity, (unsigned long long)*char_total);
    DSSS_LAUNCH("k_recv_copy", st,
                k_recv_copy<<<grid_for(n * COPY_LANES, 256), 256, 0, st>>>(a, n, L.cnt, L.cstart, recv_lcp, L.src, recv_chars,
                                                             L.longq, L.counters + 1));
    DSSS_LAUNCH("k_recv_copy_warp", st,
                k_recv_copy_warp<<<148 * 8, 256, 0, st>>>(a, L.cnt, L.cstart, recv_lcp, L.src, recv_chars, L.longq,
                                                         L.counters + 1));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

int bucket_scatter(const ExchangeLayout& L, const ArenaDev& a, uint32_t p, const uint64_t* pb,
                   const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, const uint64_t* intervals,
                   uint64_t* char_total, uint8_t* recv_chars, uint64_t recv_capacity, uint64_t* recv_char_begin,
                   uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe, uint64_t* recv_counts,
                   uint64_t* recv_offsets, uint32_t* pin, cudaStream_t st) {
    return bucket_scatter_rect(L, a, p, p, 0, pb, local_order, lcp, dp, intervals, char_total, recv_chars,
                               recv_capacity, recv_char_begin, nullptr, false, recv_lcp, recv_index, recv_pe,
                               recv_counts, recv_offsets, pin, st);
}

}  // namespace dsss
