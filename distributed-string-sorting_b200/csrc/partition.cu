// K5 — splitter sampling and partitioning: computePartition for the
// distinguishing-prefix path (src/sorter/distributed/misc.hpp:531-587, indexed
// variant :650-708).
//   sample  : per PE, nr = min(factor*(p-1), n_q) strings at local index
//             floor(i * (n_q / (nr+1))) in double arithmetic, each truncated to
//             min(length, dp) (samplingStrategies.hpp:57-89, 148-184);
//   sort    : the gathered sample with the string sort of strsort.cu, ties in
//             input order, i.e. by (PE, index) — the order IndexStringComparator
//             (misc.hpp:38-54) imposes and that RQuick's result has;
//   choose  : nr' = min(p-1, total) splitters at every (total/(nr'+1))-th
//             sorted sample (getSplitters, misc.hpp:89-135 / 137-189);
//   search  : per (PE, splitter) the reference's binary search over the PE's
//             sorted strings, which returns the first probe that compares
//             equal (binarySearch misc.hpp:310-333, binarySearchIndexed :347-374).
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "partition.cuh"
#include "strsort.cuh"

namespace dsss {

__global__ void k_sample_gather(ArenaDev a, const uint32_t* local_order, const uint32_t* dp,
                                const uint64_t* sample_lp, uint64_t m, uint64_t* soff, uint32_t* slen) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint64_t lp = sample_lp[j];
    uint64_t off;
    uint32_t len;
    str_of(a, local_order[lp], off, len);
    soff[j] = off;
    slen[j] = min(len, dp[lp]);
}

// Sign of the byte-wise comparison of two strings (scmp, stringtools.hpp:128-136).
__device__ __forceinline__ int str_cmp(const uint8_t* chars, uint64_t oa, uint32_t la, uint64_t ob, uint32_t lb) {
    for (uint32_t d = 0;; d += 8) {
        uint64_t x = key8(chars, oa, la, d), y = key8(chars, ob, lb, d);
        if (x != y) return x < y ? -1 : 1;
        if (zero_byte(x) < 8) return 0;
    }
}

// One thread per (PE, splitter): PE g of set g / p searches the set's k-th
// splitter (k < set_nspl[set]); splitters and positions are strided by p - 1.
__global__ void k_binsearch(ArenaDev a, const uint32_t* local_order, const uint64_t* pb, uint32_t npe, uint32_t p,
                            const uint32_t* set_nspl, const uint64_t* spl_off, const uint32_t* spl_len,
                            const uint64_t* spl_index, int indexed, uint64_t* pos) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = p - 1;
    if (t >= (uint64_t)npe * stride) return;
    const uint32_t g = (uint32_t)(t / stride), k = (uint32_t)(t % stride);
    const uint32_t set = g / p;
    if (k >= set_nspl[set]) return;
    const uint64_t sp = (uint64_t)set * stride + k;
    const uint64_t base = pb[g];
    uint64_t left = 0, right = pb[g + 1] - base;
    const uint64_t so = spl_off[sp];
    const uint32_t sl = spl_len[sp];
    while (left != right) {
        const uint64_t d = (right - left) / 2;
        uint64_t off;
        uint32_t len;
        str_of(a, local_order[base + left + d], off, len);
        int res = str_cmp(a.chars, off, len, so, sl);
        if (res == 0 && indexed) {
            // indexStringCompare (misc.hpp:335-345): equal bytes compare by the
            // global index, as int64 narrowed to int (both indices carry the
            // same set offset, so their difference is the set-local one).
            res = (int)(int32_t)(uint32_t)((left + d + base) - spl_index[sp]);
        }
        if (res < 0) {
            left = left + d + 1;
        } else if (res == 0) {
            pos[t] = left + d;
            return;
        } else {
            right = left + d;
        }
    }
    pos[t] = left;
}

static uint64_t max_samples(uint64_t n, uint32_t nsets, uint32_t p, uint32_t factor) {
    return std::min<uint64_t>((uint64_t)factor * (p ? p - 1 : 0) * p * nsets, n) + 1;
}

void layout_partition(Carve& c, PartitionLayout& L, uint64_t n, uint32_t p, uint32_t factor, uint32_t nsets) {
    if (nsets == 0) nsets = 1;
    const uint64_t npe = (uint64_t)nsets * p;
    uint64_t S = max_samples(n, nsets, p, factor);
    L.cap = S;
    L.sample_lp = c.take<uint64_t>(S);
    L.soff = c.take<uint64_t>(S);
    L.slen = c.take<uint32_t>(S);
    L.sorted = c.take<uint32_t>(S);
    L.slcp = c.take<uint32_t>(S);
    L.spl_off = c.take<uint64_t>(npe);
    L.spl_len = c.take<uint32_t>(npe);
    L.spl_index = c.take<uint64_t>(npe);
    L.pos = c.take<uint64_t>(npe * p + 1);
    L.pb = c.take<uint64_t>(npe + 1);
    L.set_nspl = c.take<uint32_t>(nsets);
    layout_sort(c, L.sort, S, nsets, 0);
}

int partition_sets(const PartitionLayout& L, Ctx* ctx, const ArenaDev& a, uint32_t nsets, uint32_t p,
                   const uint64_t* pb, const uint32_t* local_order, const uint32_t* dp, uint32_t sampler,
                   uint32_t factor, uint64_t* intervals, cudaStream_t st) {
    const bool indexed = sampler == DSSS_SAMPLER_INDEXED_NUM_STRINGS;
    const uint64_t npe = (uint64_t)nsets * p;
    // sample positions (host, double arithmetic as getNumberSplitter/sample_splitters)
    std::vector<uint64_t> lp, sbeg(nsets + 1, 0);
    for (uint32_t s = 0; s < nsets; ++s) {
        for (uint32_t q = 0; q < p; ++q) {
            const uint64_t g = (uint64_t)s * p + q;
            const uint64_t nq = pb[g + 1] - pb[g];
            const uint64_t nr = std::min<uint64_t>((uint64_t)factor * (p - 1), nq);
            const double dist = (double)nq / (double)(nr + 1);
            for (uint64_t i = 1; i <= nr; ++i) lp.push_back(pb[g] + (uint64_t)((double)i * dist));
        }
        sbeg[s + 1] = lp.size();
    }
    const uint64_t S = lp.size();
    if (S > L.cap) return fail(DSSS_EINVAL, "partition: sample larger than planned");
    // splitters per set: nr' = min(p - 1, the set's sample size)
    std::vector<uint32_t> nspl(nsets);
    uint64_t total_spl = 0;
    for (uint32_t s = 0; s < nsets; ++s) {
        nspl[s] = (uint32_t)std::min<uint64_t>(p - 1, sbeg[s + 1] - sbeg[s]);
        total_spl += nspl[s];
    }
    if (total_spl == 0) {
        for (uint64_t g = 0; g < npe; ++g)
            for (uint32_t r = 0; r < p; ++r) intervals[g * p + r] = r == 0 ? pb[g + 1] - pb[g] : 0;
        return DSSS_OK;
    }
    DSSS_TRY(ensure_pin(ctx, S * 16 + 64 + npe * p * 8));
    uint64_t* hpin = (uint64_t*)ctx->pin;
    std::copy(lp.begin(), lp.end(), hpin);
    DSSS_CUDA(cudaMemcpyAsync(L.sample_lp, hpin, S * 8, cudaMemcpyHostToDevice, st));
    DSSS_LAUNCH("k_sample_gather", st, k_sample_gather<<<grid_for(S, 256), 256, 0, st>>>(a, local_order, dp, L.sample_lp, S, L.soff, L.slen));
    DSSS_CUDA(cudaGetLastError());
    ArenaDev sa{a.chars, L.soff, L.slen, S};
    // sort_strings synchronises on st before reading its counts back, so the
    // sample positions copied above are consumed before hpin is reused.
    DSSS_TRY(sort_strings(L.sort, sa, S, nsets, sbeg.data(), nullptr, L.sorted, L.slcp, 0, (uint32_t*)hpin, st));
    uint32_t* hsorted = (uint32_t*)hpin;
    uint64_t* hoff = (uint64_t*)(hpin + (S + 1) / 2 + 1);
    uint32_t* hlen = (uint32_t*)(hoff + S);
    DSSS_CUDA(cudaMemcpyAsync(hsorted, L.sorted, S * 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(hoff, L.soff, S * 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(hlen, L.slen, S * 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    const uint32_t stride = p - 1;
    std::vector<uint64_t> so((uint64_t)nsets * stride), si((uint64_t)nsets * stride), pbv(pb, pb + npe + 1);
    std::vector<uint32_t> sl((uint64_t)nsets * stride);
    for (uint32_t s = 0; s < nsets; ++s) {
        if (!nspl[s]) continue;
        const uint64_t sd = (sbeg[s + 1] - sbeg[s]) / (nspl[s] + 1);
        for (uint64_t k = 1; k <= nspl[s]; ++k) {
            const uint32_t sid = hsorted[sbeg[s] + k * sd];  // sorted ids are sample positions
            so[(uint64_t)s * stride + k - 1] = hoff[sid];
            sl[(uint64_t)s * stride + k - 1] = hlen[sid];
            si[(uint64_t)s * stride + k - 1] = lp[sid];
        }
    }
    DSSS_CUDA(cudaMemcpyAsync(L.spl_off, so.data(), so.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.spl_len, sl.data(), sl.size() * 4, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.spl_index, si.data(), si.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.pb, pbv.data(), (npe + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.set_nspl, nspl.data(), nsets * 4, cudaMemcpyHostToDevice, st));
    const uint64_t tasks = npe * stride;
    DSSS_LAUNCH("k_binsearch", st, k_binsearch<<<grid_for(tasks, 128), 128, 0, st>>>(a, local_order, L.pb, (uint32_t)npe, p, L.set_nspl,
                                                                  L.spl_off, L.spl_len, L.spl_index, indexed ? 1 : 0, L.pos));
    DSSS_CUDA(cudaGetLastError());
    std::vector<uint64_t> pos(tasks);
    DSSS_CUDA(cudaMemcpyAsync(pos.data(), L.pos, tasks * 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    // compute_interval_binary (misc.hpp:376-395): differences of the positions
    for (uint64_t g = 0; g < npe; ++g) {
        const uint32_t ns = nspl[g / p];
        uint64_t prev = 0;
        for (uint32_t r = 0; r < p; ++r) {
            uint64_t cur = r < ns ? pos[g * stride + r] : pb[g + 1] - pb[g];
            intervals[g * p + r] = cur - prev;
            prev = cur;
        }
    }
    return DSSS_OK;
}

int partition_pes(const PartitionLayout& L, Ctx* ctx, const ArenaDev& a, uint32_t p, const uint64_t* pb,
                  const uint32_t* local_order, const uint32_t* dp, uint32_t sampler, uint32_t factor,
                  uint64_t* intervals, cudaStream_t st) {
    return partition_sets(L, ctx, a, 1, p, pb, local_order, dp, sampler, factor, intervals, st);
}

// ---- PEs on several GPUs: search splitters gathered from every GPU ----
__device__ __forceinline__ int str_cmp2(const uint8_t* ca, uint64_t oa, uint32_t la, const uint8_t* cb, uint64_t ob,
                                        uint32_t lb) {
    for (uint32_t d = 0;; d += 8) {
        uint64_t x = key8(ca, oa, la, d), y = key8(cb, ob, lb, d);
        if (x != y) return x < y ? -1 : 1;
        if (zero_byte(x) < 8) return 0;
    }
}

// One thread per (local PE g, splitter k): the reference's binary search of
// PE g's sorted strings for splitter k; goff[g]: the global index of PE g's
// first string (indexed compare).
__global__ void k_binsearch_ext(ArenaDev a, const uint32_t* local_order, const uint64_t* pb, const uint64_t* goff,
                                uint32_t npe, ArenaDev sp, const uint64_t* spl_index, int indexed, uint64_t* pos) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nspl = (uint32_t)sp.n;
    if (t >= (uint64_t)npe * nspl) return;
    const uint32_t g = (uint32_t)(t / nspl), k = (uint32_t)(t % nspl);
    const uint64_t base = pb[g];
    uint64_t left = 0, right = pb[g + 1] - base;
    uint64_t so;
    uint32_t sl;
    str_of(sp, k, so, sl);
    while (left != right) {
        const uint64_t d = (right - left) / 2;
        uint64_t off;
        uint32_t len;
        str_of(a, local_order[base + left + d], off, len);
        int res = str_cmp2(a.chars, off, len, sp.chars, so, sl);
        if (res == 0 && indexed) res = (int)(int32_t)(uint32_t)((left + d + goff[g]) - spl_index[k]);
        if (res < 0) {
            left = left + d + 1;
        } else if (res == 0) {
            pos[t] = left + d;
            return;
        } else {
            right = left + d;
        }
    }
    pos[t] = left;
}

int partition_search(Ctx* ctx, const ArenaDev& a, uint32_t p_local, const uint64_t* pb, const uint32_t* local_order,
                     const ArenaDev& sp, const uint64_t* spl_index_host, uint32_t p_global, const uint64_t* goff_host,
                     int indexed, uint64_t* intervals, cudaStream_t st) {
    const uint32_t nspl = (uint32_t)sp.n;
    if (nspl + 1 > p_global) return fail(DSSS_EINVAL, "%u splitters for %u PEs", nspl, p_global);
    const uint64_t tasks = (uint64_t)p_local * nspl;
    Carve sz(nullptr);
    sz.take<uint64_t>(p_local + 1);
    sz.take<uint64_t>(p_local + 1);
    sz.take<uint64_t>(nspl + 1);
    sz.take<uint64_t>(tasks + 1);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    Carve c(ctx->ws);
    uint64_t* d_pb = c.take<uint64_t>(p_local + 1);
    uint64_t* d_goff = c.take<uint64_t>(p_local + 1);
    uint64_t* d_si = c.take<uint64_t>(nspl + 1);
    uint64_t* d_pos = c.take<uint64_t>(tasks + 1);
    std::vector<uint64_t> gv(p_local + 1, 0), siv(nspl + 1, 0), pos(tasks);
    if (indexed) {
        for (uint32_t g = 0; g < p_local; ++g) gv[g] = goff_host[g];
        for (uint32_t k = 0; k < nspl; ++k) siv[k] = spl_index_host[k];
    }
    if (tasks) {
        DSSS_CUDA(cudaMemcpyAsync(d_pb, pb, (p_local + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(d_goff, gv.data(), (p_local + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(d_si, siv.data(), (nspl + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_binsearch", st,
                    k_binsearch_ext<<<grid_for(tasks, 128), 128, 0, st>>>(a, local_order, d_pb, d_goff, p_local, sp,
                                                                          d_si, indexed, d_pos));
        DSSS_CUDA(cudaGetLastError());
        DSSS_CUDA(cudaMemcpyAsync(pos.data(), d_pos, tasks * 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
    }
    // compute_interval_binary (misc.hpp:376-395)
    for (uint32_t g = 0; g < p_local; ++g) {
        uint64_t prev = 0;
        for (uint32_t r = 0; r < p_global; ++r) {
            const uint64_t cur = r < nspl ? pos[(uint64_t)g * nspl + r] : pb[g + 1] - pb[g];
            intervals[(uint64_t)g * p_global + r] = cur - prev;
            prev = cur;
        }
    }
    return DSSS_OK;
}

}  // namespace dsss
