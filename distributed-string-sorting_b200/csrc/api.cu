// C ABI entry points: the full prefix-doubling path and one entry per stage.
//
// The full path (dsss_pd_sort) is laid out for one GPU holding every PE:
//   1. one string sort of all n strings (K3, LCP as by-product);
//   2. distinguishing-prefix rounds over that global order (K1/K2) — the
//      result per string does not depend on the PE split;
//   3. stable multisplit by PE of the global order gives each PE's local sorted
//      order (a subsequence of a sorted sequence is sorted), i.e. exactly what
//      radixsort_CI3 produces per PE (prefix_doubling.hpp:228);
//   4. partition (K5) on those local orders;
//   5. every string's bucket follows from its PE and local index; a stable
//      multisplit of the global order by bucket is each receiving PE's merged
//      sequence — what AllToAllStringImplPrefixDoubling + choose_merge deliver
//      (prefix_doubling.hpp:254-281) — with (local index, PE) as the
//      permutation (:282-290) and merged LCPs taken from the global LCPs.
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include "dp.cuh"
#include "exchange.cuh"
#include "internal.cuh"
#include "merge.cuh"
#include "partition.cuh"
#include "pd.cuh"
#include "strsort.cuh"
#include "util.cuh"

namespace dsss {

static int check_parts(uint32_t p, const uint64_t* pb, uint64_t n) {
    if (p == 0) return fail(DSSS_EINVAL, "p must be >= 1");
    if (!pb) return fail(DSSS_EINVAL, "part_begin is NULL");
    if (pb[0] != 0 || pb[p] != n) return fail(DSSS_EINVAL, "part_begin must start at 0 and end at n");
    for (uint32_t q = 0; q < p; ++q)
        if (pb[q + 1] < pb[q]) return fail(DSSS_EINVAL, "part_begin must be non-decreasing");
    return DSSS_OK;
}

static ArenaDev view(const dsss_arena* a) { return ArenaDev{a->chars, a->offsets, a->lengths, a->n}; }

static uint32_t factor_of(const dsss_opts* o) { return (o && o->sampling_factor) ? o->sampling_factor : 2; }
static uint32_t sampler_of(const dsss_opts* o) { return o ? o->sampler : DSSS_SAMPLER_NUM_STRINGS; }
static uint32_t smallmax_of(const dsss_opts* o) { return o ? o->small_sort_max : 0; }

// PE of every sorted position: the q with pb[q] <= ord[g] < pb[q + 1] in a
// shared-memory copy of the PE bounds (npe + 1 <= 1025 entries), PE_IPT
// positions per thread with their ids loaded before the lookups.  The first
// guess is the PE that equal parts would give (id * p / n), moved by up to
// two steps; a guess that is still off (PEs of very uneven sizes) falls back
// to a binary search.
constexpr int PE_NT = 256, PE_IPT = 8;
__global__ void __launch_bounds__(PE_NT) k_pe_of(const uint32_t* ord, uint64_t n, const uint64_t* pb, uint32_t p,
                                                 uint32_t* pe) {
    extern __shared__ unsigned long long spb[];
    for (uint32_t q = threadIdx.x; q <= p; q += PE_NT) spb[q] = pb[q];
    const uint64_t g0 = (uint64_t)blockIdx.x * (PE_NT * PE_IPT) + threadIdx.x;
    uint32_t s[PE_IPT];
#pragma unroll
    for (int j = 0; j < PE_IPT; ++j) {
        const uint64_t g = g0 + (uint64_t)j * PE_NT;
        s[j] = g < n ? ord[g] : 0u;
    }
    __syncthreads();
    const float scale = (float)p / (float)(spb[p] ? spb[p] : 1ull);
    uint32_t q[PE_IPT];
#pragma unroll
    for (int j = 0; j < PE_IPT; ++j) q[j] = min(p - 1, (uint32_t)((float)s[j] * scale));
#pragma unroll
    for (int step = 0; step < 2; ++step) {
#pragma unroll
        for (int j = 0; j < PE_IPT; ++j) {
            if (spb[q[j]] > s[j]) --q[j];                        // q[j] > 0 here: spb[0] = 0
            else if (spb[q[j] + 1] <= s[j]) ++q[j];              // q[j] + 1 < p here: spb[p] = n > s
        }
    }
#pragma unroll
    for (int j = 0; j < PE_IPT; ++j) {
        const uint64_t g = g0 + (uint64_t)j * PE_NT;
        if (g >= n) continue;
        uint32_t r = q[j];
        if (spb[r] > s[j] || spb[r + 1] <= s[j]) {  // still off: the last r < p with pb[r] <= s
            r = 0;
            for (uint32_t st = 1u << (31 - __clz(p | 1u)); st; st >>= 1)
                if (r + st < p && spb[r + st] <= s[j]) r += st;
        }
        pe[g] = r;
    }
}

static int launch_pe_of(const uint32_t* ord, uint64_t n, const uint64_t* pb, uint32_t p, uint32_t* pe,
                        cudaStream_t st) {
    const uint64_t per = (uint64_t)PE_NT * PE_IPT;
    DSSS_LAUNCH("k_pe_of", st,
                k_pe_of<<<(unsigned)((n + per - 1) / per), PE_NT, (p + 1) * sizeof(unsigned long long), st>>>(
                    ord, n, pb, p, pe));
    return DSSS_OK;
}

// Receiving PE of every string: set s's PE q sends local positions
// [bounds[(s*p+q)*(p+1) + r], … + r + 1) to the set's PE r; buckets are
// numbered s*p + r.  src is q's global PE number, li the string's index in
// q's local order; B is the bound table (u64 in global memory, or a u32 copy
// in shared memory).
template <typename B>
__device__ __forceinline__ uint32_t bucket_of(const B* bounds, uint32_t p, uint32_t src, uint32_t li) {
    const B* b = bounds + (uint64_t)src * (p + 1);
    uint32_t lo = 0;  // the last r < p with b[r] <= li (b[0] = 0), in fixed steps
    for (uint32_t step = 1u << (31 - __clz(p | 1u)); step; step >>= 1) {
        const uint32_t m = lo + step;
        if (m < p && b[m] <= li) lo = m;
    }
    return (src / p) * p + lo;
}

// k_bucket_of plus, for the common case, the merged sequences themselves: when
// the buckets never decrease along the global order (no equal strings that two
// PEs cut on different sides of a splitter), the stable partition by bucket
// is the identity, so position g of the merged sequences is global position g:
// its (local index, sender PE) and, unless it starts a receiving PE's run, the
// global LCP.  *viol is set when some bucket decreases; the caller then runs
// the multisplit, which rewrites every output (bucket, when given, receives
// every position's bucket for it).  BD_IPT positions per thread, their inputs
// loaded before the searches; with SMEM the bound table is searched in a u32
// copy in shared memory; each position's predecessor bucket comes from the
// tile's bucket row in shared memory.
constexpr int BD_NT = 256, BD_IPT = 8, BD_TILE = BD_NT * BD_IPT;
constexpr uint32_t BD_SMEM_BOUNDS = 8192;  // bound entries kept in shared memory (32 KiB)
template <bool SMEM>
__global__ void __launch_bounds__(BD_NT, 4) k_bucket_direct(const uint32_t* pe, const uint32_t* g2l,
                                                         const uint64_t* bounds, uint32_t p, uint32_t npe, uint64_t n,
                                                         int local_pe, const uint32_t* lcpg, uint32_t* bucket,
                                                         uint32_t* pe_local, uint32_t* perm_index, uint32_t* perm_pe,
                                                         uint32_t* merged, uint32_t* viol) {
    extern __shared__ uint32_t sbd[];
    uint32_t* sb = sbd;                  // the tile's buckets, after the one of the position before it
    uint32_t* tab = sbd + BD_TILE + 1;   // SMEM: npe * (p + 1) bounds
    const uint64_t t0 = (uint64_t)blockIdx.x * BD_TILE;
    if (SMEM)
        for (uint32_t k = threadIdx.x; k < npe * (p + 1); k += BD_NT) tab[k] = (uint32_t)bounds[k];
    uint32_t src[BD_IPT], li[BD_IPT], lc[BD_IPT];
#pragma unroll
    for (int j = 0; j < BD_IPT; ++j) {
        const uint64_t g = t0 + (uint64_t)j * BD_NT + threadIdx.x;
        const bool v = g < n;
        src[j] = v ? pe[g] : 0u;
        li[j] = v ? g2l[g] : 0u;
        lc[j] = v && merged ? lcpg[g] : 0u;
    }
    __syncthreads();
    // the BD_IPT searches interleaved, in the fixed steps of bucket_of
    uint32_t bk[BD_IPT];
#pragma unroll
    for (int j = 0; j < BD_IPT; ++j) bk[j] = 0;
    for (uint32_t step = 1u << (31 - __clz(p | 1u)); step; step >>= 1) {
#pragma unroll
        for (int j = 0; j < BD_IPT; ++j) {
            const uint32_t m = bk[j] + step;
            if (m < p) {
                const bool le = SMEM ? tab[src[j] * (p + 1) + m] <= li[j]
                                     : bounds[(uint64_t)src[j] * (p + 1) + m] <= li[j];
                if (le) bk[j] = m;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < BD_IPT; ++j) {
        bk[j] += (src[j] / p) * p;
        sb[1 + j * BD_NT + threadIdx.x] = bk[j];
    }
    if (threadIdx.x == 0) {
        uint32_t b = 0xFFFFFFFFu;
        if (t0 && t0 <= n) {
            const uint32_t s0 = pe[t0 - 1], l0 = g2l[t0 - 1];
            b = SMEM ? bucket_of(tab, p, s0, l0) : bucket_of(bounds, p, s0, l0);
        }
        sb[0] = b;
    }
    __syncthreads();
    bool bad = false;
#pragma unroll
    for (int j = 0; j < BD_IPT; ++j) {
        const uint64_t g = t0 + (uint64_t)j * BD_NT + threadIdx.x;
        if (g >= n) continue;
        const uint32_t b = bk[j], bp = sb[j * BD_NT + threadIdx.x];
        if (g && bp > b) bad = true;
        const uint32_t ql = src[j] - (src[j] / p) * p;
        if (bucket) bucket[g] = b;
        if (pe_local) pe_local[g] = ql;
        perm_index[g] = li[j];
        perm_pe[g] = local_pe ? ql : src[j];
        if (merged) merged[g] = (g == 0 || bp != b) ? 0u : lc[j];
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(viol, 1u);
}

static int launch_bucket_direct(const uint32_t* pe, const uint32_t* g2l, const uint64_t* bounds, uint32_t p,
                                uint32_t npe, uint64_t n, int local_pe, const uint32_t* lcpg, uint32_t* bucket,
                                uint32_t* pe_local, uint32_t* perm_index, uint32_t* perm_pe, uint32_t* merged,
                                uint32_t* viol, cudaStream_t st) {
    const unsigned grid = (unsigned)((n + BD_TILE - 1) / BD_TILE);
    const uint64_t entries = (uint64_t)npe * (p + 1);
    if (entries <= BD_SMEM_BOUNDS) {
        const size_t sm = (BD_TILE + 1 + entries) * sizeof(uint32_t);
        DSSS_LAUNCH("k_bucket_direct", st,
                    k_bucket_direct<true><<<grid, BD_NT, sm, st>>>(pe, g2l, bounds, p, npe, n, local_pe, lcpg, bucket,
                                                                   pe_local, perm_index, perm_pe, merged, viol));
    } else {
        const size_t sm = (BD_TILE + 1) * sizeof(uint32_t);
        DSSS_LAUNCH("k_bucket_direct", st,
                    k_bucket_direct<false><<<grid, BD_NT, sm, st>>>(pe, g2l, bounds, p, npe, n, local_pe, lcpg,
                                                                    bucket, pe_local, perm_index, perm_pe, merged,
                                                                    viol));
    }
    return DSSS_OK;
}

__global__ void k_merged_lcp(const uint32_t* out2g, const uint32_t* lcpg, const uint64_t* recv_begin, uint32_t p,
                             uint64_t n, uint32_t* merged) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    uint32_t lo = 0, hi = p;  // is o the first string of some PE's merged run?
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (recv_begin[mid] <= o) lo = mid;
        else hi = mid;
    }
    bool first = false;
    for (uint32_t r = lo; r < p && recv_begin[r] <= o; ++r)
        if (recv_begin[r] == o) { first = true; break; }
    if (first) { merged[o] = 0; return; }
    const uint32_t g = out2g[o], gp = out2g[o - 1];
    uint32_t l = 0xFFFFFFFFu;
    for (uint32_t x = gp + 1; x <= g; ++x) l = min(l, lcpg[x]);  // LCP over the skipped run
    merged[o] = l;
}

__global__ void k_zero_starts(uint32_t* a, const uint64_t* pb, uint32_t p) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < p && pb[q] < pb[q + 1]) a[pb[q]] = 0;
}

struct PdLayout {
    ulonglong2* handles;
    uint32_t *ord, *lcp, *dpg, *pe, *g2l, *tmp, *out2g, *pel, *nlong, *err, *viol;
    uint64_t *pb, *bounds, *recv_begin;
    void* ms;
    SortLayout sort;
    DpLayout dp;
    PartitionLayout part;
    unsigned long long* rdig;  // prefix hashes at the first schedule depths, from the sort's first pass
};

// n strings in nsets sets of p PEs each.
static void layout_pd(Carve& c, PdLayout& L, uint64_t n, uint32_t nsets, uint32_t p, uint32_t factor,
                      uint32_t small_max) {
    uint64_t N = n ? n : 1;
    const uint64_t npe = (uint64_t)nsets * p;
    L.handles = c.take<ulonglong2>(N);
    L.ord = c.take<uint32_t>(N);
    L.lcp = c.take<uint32_t>(N);
    L.dpg = c.take<uint32_t>(N);
    L.pe = c.take<uint32_t>(N);
    L.g2l = c.take<uint32_t>(N);
    L.tmp = c.take<uint32_t>(N);
    L.out2g = c.take<uint32_t>(N);
    L.pel = nsets > 1 ? c.take<uint32_t>(N) : nullptr;
    L.nlong = c.take<uint32_t>(1);
    L.err = c.take<uint32_t>(1);
    L.viol = c.take<uint32_t>(1);
    L.pb = c.take<uint64_t>(npe + 1);
    L.bounds = c.take<uint64_t>(npe * (p + 1));
    L.recv_begin = c.take<uint64_t>(npe + 1);
    L.ms = c.take<unsigned char>(multisplit_scratch_bytes(N, (uint32_t)npe));
    layout_sort(c, L.sort, N, nsets, small_max);
    layout_dp(c, L.dp, N, nsets);
    layout_partition(c, L.part, N, p, factor, nsets);
    // decided by a value both carving passes see (the sizing pass hands out
    // null pointers)
    L.rdig = L.dp.digest_share ? c.take<unsigned long long>(ROOT_DIGESTS * N) : nullptr;
}

// The fused path over nsets independent string sets of p PEs each (PE q of
// set s = part_begin[s*p + q] .. part_begin[s*p + q + 1]); every set's result
// is the one a call on that set alone gives.  Per-string outputs keep the
// arena's positions (set s's merged sequences fill the positions of its
// strings), intervals and recv_counts are per set, one after the other.
uint64_t pd_scratch_bytes(uint64_t n, uint32_t nsets, uint32_t p, const dsss_opts* opts) {
    Carve sz(nullptr);
    PdLayout L;
    layout_pd(sz, L, n, nsets, p, factor_of(opts), smallmax_of(opts));
    return sz.used;
}

int pd_sort_dev(Ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p, const uint64_t* pb,
                const dsss_opts* opts, dsss_pd_result* out, cudaStream_t st) {
    DSSS_TRY(check_arena(in));
    if (nsets == 0) return fail(DSSS_EINVAL, "nsets must be >= 1");
    if (p == 0) return fail(DSSS_EINVAL, "p must be >= 1");
    if ((uint64_t)nsets * p > MAX_SPLIT_BUCKETS)
        return fail(DSSS_ENOTSUP, "nsets * p > %u PEs per GPU is not supported", MAX_SPLIT_BUCKETS);
    const uint32_t npe = nsets * p;
    DSSS_TRY(check_parts(npe, pb, in->n));
    if (!out || !out->local_order || !out->recv_counts) return fail(DSSS_EINVAL, "result arrays missing");
    if (p > 1 && (!out->dp || !out->intervals || !out->perm_index || !out->perm_pe))
        return fail(DSSS_EINVAL, "result arrays missing");
    const uint64_t n = in->n;
    const uint32_t factor = factor_of(opts), smax = smallmax_of(opts);
    const bool want_local_lcp = opts && (opts->flags & DSSS_FLAG_LOCAL_LCP) && out->local_lcp;
    Carve sz(nullptr);
    PdLayout L;
    layout_pd(sz, L, n, nsets, p, factor, smax);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_pd(c, L, n, nsets, p, factor, smax);
    uint32_t* pin = (uint32_t*)ctx->pin;  // re-read after any call that may grow it
    ArenaDev a = view(in);
    if (n == 0) {
        for (uint32_t r = 0; r < npe; ++r) out->recv_counts[r] = 0;
        if (p > 1)
            for (uint64_t k = 0; k < (uint64_t)npe * p; ++k) out->intervals[k] = 0;
        return DSSS_OK;
    }
    std::vector<uint64_t> set_begin(nsets + 1);
    for (uint32_t s = 0; s <= nsets; ++s) set_begin[s] = pb[(uint64_t)s * p];
    make_handles(a, L.handles, st);
    a.h = L.handles;
    DSSS_CUDA(cudaMemsetAsync(L.err, 0, sizeof(uint32_t), st));
    // 1. one sort per set, all sets in one segmented sort
    uint32_t rdig_mask = 0;
    {
        StageTimer t("stage:sort", st);
        DSSS_TRY(sort_strings(L.sort, a, n, nsets, set_begin.data(), nullptr, L.ord, L.lcp, smax, pin, st,
                              p > 1 ? L.rdig : nullptr, &rdig_mask));
    }
    if (p == 1) {  // prefix_doubling.hpp:236: one PE sorts locally and returns no permutation
        DSSS_CUDA(cudaMemcpyAsync(out->local_order, L.ord, n * 4, cudaMemcpyDeviceToDevice, st));
        if (want_local_lcp) DSSS_CUDA(cudaMemcpyAsync(out->local_lcp, L.lcp, n * 4, cudaMemcpyDeviceToDevice, st));
        for (uint32_t r = 0; r < npe; ++r) out->recv_counts[r] = 0;
        return DSSS_OK;
    }
    // 2. distinguishing prefixes over each set's sorted order
    {
        StageTimer t("stage:dp", st);
        DSSS_TRY(dp_rounds(L.dp, a, n, L.ord, L.lcp, L.dpg, nullptr, 0, nullptr, pin, st, nsets, set_begin.data(),
                           rdig_mask ? L.rdig : nullptr, rdig_mask));
    }
    // 3. local orders per PE
    StageTimer t_local("stage:local", st);
    DSSS_CUDA(cudaMemcpyAsync(L.pb, pb, (npe + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_TRY(launch_pe_of(L.ord, n, L.pb, npe, L.pe, st));
    {
        // local order and DP per PE: out[dest] = (string id, dp); g2l = rank inside the PE
        const uint32_t* in[2] = {L.ord, L.dpg};
        uint32_t* outs[2] = {out->local_order, out->dp};
        DSSS_TRY(multisplit_payload(L.pe, n, npe, 2, in, outs, L.g2l, L.err, L.ms, st));
    }
    DSSS_CUDA(cudaGetLastError());
    t_local.end();
    // 4. partition
    {
        StageTimer t("stage:partition", st);
        DSSS_TRY(partition_sets(L.part, ctx, a, nsets, p, pb, out->local_order, out->dp, sampler_of(opts), factor,
                                out->intervals, st));
    }
    StageTimer t_merge("stage:merge", st);
    // 5. buckets and the merged sequences; receiving PE (s, r) is bucket s*p + r
    std::vector<uint64_t> bounds((uint64_t)npe * (p + 1)), recv(npe + 1, 0);
    for (uint32_t g = 0; g < npe; ++g) {
        const uint32_t s = g / p;
        bounds[(uint64_t)g * (p + 1)] = 0;
        for (uint32_t r = 0; r < p; ++r) {
            uint64_t v = out->intervals[(uint64_t)g * p + r];
            bounds[(uint64_t)g * (p + 1) + r + 1] = bounds[(uint64_t)g * (p + 1) + r] + v;
            recv[(uint64_t)s * p + r + 1] += v;
        }
    }
    for (uint32_t r = 0; r < npe; ++r) {
        out->recv_counts[r] = recv[r + 1];
        recv[r + 1] += recv[r];
    }
    DSSS_CUDA(cudaMemcpyAsync(L.bounds, bounds.data(), bounds.size() * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(L.recv_begin, recv.data(), (npe + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemsetAsync(L.viol, 0, sizeof(uint32_t), st));
    DSSS_TRY(launch_bucket_direct(L.pe, L.g2l, L.bounds, p, npe, n, nsets > 1, L.lcp, nullptr, L.pel,
                                  out->perm_index, out->perm_pe, out->merged_lcp, L.viol, st));
    pin = (uint32_t*)ctx->pin;  // the partition step may have grown the staging buffer
    DSSS_CUDA(cudaMemcpyAsync(pin, L.viol, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) {
        // every position's bucket for the multisplit (the outputs are rewritten by it)
        DSSS_TRY(launch_bucket_direct(L.pe, L.g2l, L.bounds, p, npe, n, nsets > 1, L.lcp, L.tmp, L.pel,
                                      out->perm_index, out->perm_pe, nullptr, L.viol, st));
        // merged sequences: (index in sender's local order, sender PE, global position)
        const uint32_t* in[3] = {L.g2l, nsets > 1 ? L.pel : L.pe, nullptr};
        uint32_t* outs[3] = {out->perm_index, out->perm_pe, L.out2g};
        DSSS_TRY(multisplit_payload(L.tmp, n, npe, 3, in, outs, nullptr, L.err, L.ms, st));
        if (out->merged_lcp)
            DSSS_LAUNCH("k_merged_lcp", st,
                        k_merged_lcp<<<grid_for(n, 256), 256, 0, st>>>(L.out2g, L.lcp, L.recv_begin, npe, n,
                                                                      out->merged_lcp));
    }
    if (want_local_lcp) {
        DSSS_TRY(adjacent_lcp(a, out->local_order, n, out->local_lcp, L.tmp, L.nlong, st));
        DSSS_LAUNCH("k_zero_starts", st, k_zero_starts<<<grid_for(npe, 128), 128, 0, st>>>(out->local_lcp, L.pb, npe));
    }
    DSSS_CUDA(cudaGetLastError());
    // The host vectors above were copied asynchronously; finish before they go.
    pin = (uint32_t*)ctx->pin;  // the partition step may have grown the staging buffer
    DSSS_CUDA(cudaMemcpyAsync(pin, L.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) return fail(DSSS_EDEVICE, "pd sort: internal consistency guard tripped");
    return DSSS_OK;
}

// ------------------------------------------------------- merge-sort path ----
// DistributedMergeSort::sort on one GPU holding every PE: the global sort, the
// local orders (multisplit by PE) and their LCP arrays, getAvgLcp, the
// partition with samples cut to 200 (avg + 5) bytes, then the receiving PEs'
// sequences as a projection of the global order (written directly, or by the
// multisplit by bucket when ties cross a splitter) and their strings copied
// out whole.

__global__ void k_sum_u32_to_u64(const uint32_t* v, uint64_t n, unsigned long long* total) {
    unsigned long long s = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += v[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

__global__ void k_fill_u32(uint32_t* a, uint64_t n, uint32_t v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// Input index, source offset and length (+ 1 for the scan) of every output
// string: the copy then reads its string's place sequentially instead of
// gathering it again.
__global__ void k_ms_source(const uint32_t* local_order, const uint64_t* pb, const uint32_t* perm_index,
                            const uint32_t* perm_pe, ArenaDev a, uint64_t n, uint32_t* source, uint32_t* lengths,
                            uint32_t* len1, uint64_t* src_off) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const uint32_t id = perm_pe ? local_order[pb[perm_pe[o]] + perm_index[o]] : local_order[o];
    uint64_t off;
    uint32_t len;
    str_of(a, id, off, len);
    source[o] = id;
    lengths[o] = len;
    len1[o] = len + 1;
    src_off[o] = off;
}

// Whole output strings and their NULs, MS_COPY_LANES lanes per string
// (copy_words16: aligned 16-byte stores, 3.5% faster on B200 than
// copy_words' 8-byte ones, which the knob copy_word = 8 selects; 8 lanes
// measured faster than 4 or 32).
constexpr uint32_t MS_COPY_LANES = 8;
template <uint32_t W>
__global__ void k_ms_copy(const uint8_t* chars, const uint64_t* src_off, const uint32_t* lengths,
                          const uint64_t* out_off, uint64_t n, uint8_t* out) {
    const uint64_t o = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / MS_COPY_LANES;
    const uint32_t lane = threadIdx.x % MS_COPY_LANES;
    if (o >= n) return;
    const uint32_t len = lengths[o];
    uint8_t* dst = out + out_off[o];
    if (W == 16) copy_words16<MS_COPY_LANES>(dst, chars + src_off[o], len, lane);
    else copy_words<MS_COPY_LANES>(dst, chars + src_off[o], len, lane);
    if (lane == 0) dst[len] = 0;
}

static int launch_ms_copy(const uint8_t* chars, const uint64_t* src_off, const uint32_t* lengths,
                          const uint64_t* out_off, uint64_t n, uint8_t* out, cudaStream_t st) {
    const unsigned grid = grid_for(n * MS_COPY_LANES, 256);
    if (tune(TUNE_COPY_WORD) == 16)
        DSSS_LAUNCH("k_ms_copy", st, k_ms_copy<16><<<grid, 256, 0, st>>>(chars, src_off, lengths, out_off, n, out));
    else
        DSSS_LAUNCH("k_ms_copy", st, k_ms_copy<8><<<grid, 256, 0, st>>>(chars, src_off, lengths, out_off, n, out));
    return DSSS_OK;
}

static int ms_sort_dev(Ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* pb, const dsss_opts* opts,
                       dsss_ms_result* out, cudaStream_t st) {
    DSSS_TRY(check_arena(in));
    if (p == 0) return fail(DSSS_EINVAL, "p must be >= 1");
    if (p > MAX_SPLIT_BUCKETS) return fail(DSSS_ENOTSUP, "p > %u PEs per GPU is not supported", MAX_SPLIT_BUCKETS);
    DSSS_TRY(check_parts(p, pb, in->n));
    if (!out || !out->local_order || !out->recv_counts || !out->intervals || !out->offsets || !out->lengths ||
        !out->lcp || (in->n && !out->chars))
        return fail(DSSS_EINVAL, "result arrays missing");
    if (opts && opts->sampler != DSSS_SAMPLER_NUM_STRINGS)
        return fail(DSSS_ENOTSUP, "the merge-sort path samples with SampleSplittersNumStringsPolicy only");
    const uint64_t n = in->n;
    const uint32_t factor = 2, smax = smallmax_of(opts);  // computePartition(..., 2): misc.hpp call in :238
    const uint64_t N = n ? n : 1;
    Carve sz(nullptr);
    PdLayout L;
    layout_pd(sz, L, n, 1, p, factor, smax);
    uint32_t* src_tmp = sz.take<uint32_t>(N);
    uint32_t* len1 = sz.take<uint32_t>(N);
    uint64_t* srcoff = sz.take<uint64_t>(N);
    unsigned long long* total = sz.take<unsigned long long>(2);
    void* scan = sz.take<unsigned char>(scan_scratch_bytes(N));
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_pd(c, L, n, 1, p, factor, smax);
    src_tmp = c.take<uint32_t>(N);
    len1 = c.take<uint32_t>(N);
    srcoff = c.take<uint64_t>(N);
    total = c.take<unsigned long long>(2);
    scan = c.take<unsigned char>(scan_scratch_bytes(N));
    uint32_t* source = out->source ? out->source : src_tmp;
    out->avg_lcp = 0;
    if (n == 0) {
        for (uint32_t r = 0; r < p; ++r) out->recv_counts[r] = 0;
        for (uint64_t k = 0; k < (uint64_t)p * p; ++k) out->intervals[k] = 0;
        return DSSS_OK;
    }
    ArenaDev a = view(in);
    make_handles(a, L.handles, st);
    a.h = L.handles;
    uint32_t* pin = (uint32_t*)ctx->pin;
    DSSS_CUDA(cudaMemsetAsync(L.err, 0, sizeof(uint32_t), st));
    DSSS_CUDA(cudaMemsetAsync(total, 0, 2 * sizeof(unsigned long long), st));
    const uint64_t set_begin[2] = {0, n};
    {
        StageTimer t("stage:sort", st);
        DSSS_TRY(sort_strings(L.sort, a, n, 1, set_begin, nullptr, L.ord, L.lcp, smax, pin, st));
    }
    // local orders per PE and their LCP arrays (0 at each PE start)
    StageTimer t_local("stage:local", st);
    DSSS_CUDA(cudaMemcpyAsync(L.pb, pb, (p + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_TRY(launch_pe_of(L.ord, n, L.pb, p, L.pe, st));
    {
        const uint32_t* ins[1] = {L.ord};
        uint32_t* outs[1] = {out->local_order};
        DSSS_TRY(multisplit_payload(L.pe, n, p, 1, ins, outs, L.g2l, L.err, L.ms, st));
    }
    // L.dpg holds the local LCPs, then the sample cut
    DSSS_TRY(adjacent_lcp(a, out->local_order, n, L.dpg, L.tmp, L.nlong, st));
    DSSS_LAUNCH("k_zero_starts", st, k_zero_starts<<<grid_for(p, 128), 128, 0, st>>>(L.dpg, L.pb, p));
    DSSS_LAUNCH("k_sum_u32_to_u64", st, k_sum_u32_to_u64<<<148 * 4, 256, 0, st>>>(L.dpg, n, total));
    pin = (uint32_t*)ctx->pin;
    DSSS_CUDA(cudaMemcpyAsync(pin, total, 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    const uint64_t avg = *(const uint64_t*)pin / n;  // getAvgLcp (misc.hpp:68-87)
    out->avg_lcp = avg;
    t_local.end();
    if (p == 1) {  // lcp_aware_number_string_splitting.hpp:230-232: the local sort is the result
        out->intervals[0] = n;
        out->recv_counts[0] = n;
        StageTimer t("stage:merge", st);
        DSSS_CUDA(cudaMemcpyAsync(out->lcp, L.dpg, n * 4, cudaMemcpyDeviceToDevice, st));
        DSSS_LAUNCH("k_ms_source", st,
                    k_ms_source<<<grid_for(n, 256), 256, 0, st>>>(out->local_order, L.pb, nullptr, nullptr, a, n,
                                                                 source, out->lengths, len1, srcoff));
    } else {
        {
            StageTimer t("stage:partition", st);
            const uint64_t cut = 2 * (100 * (avg + 5));  // misc.hpp:488 on 100 * globalLcpAvg (:238)
            DSSS_LAUNCH("k_fill_u32", st,
                        k_fill_u32<<<grid_for(n, 256), 256, 0, st>>>(L.dpg, n, cut > 0xFFFFFFFFull ? 0xFFFFFFFFu
                                                                                                 : (uint32_t)cut));
            DSSS_TRY(partition_sets(L.part, ctx, a, 1, p, pb, out->local_order, L.dpg, DSSS_SAMPLER_NUM_STRINGS,
                                    factor, out->intervals, st));
        }
        StageTimer t_merge("stage:merge", st);
        std::vector<uint64_t> bounds((uint64_t)p * (p + 1)), recv(p + 1, 0);
        for (uint32_t q = 0; q < p; ++q) {
            bounds[(uint64_t)q * (p + 1)] = 0;
            for (uint32_t r = 0; r < p; ++r) {
                const uint64_t v = out->intervals[(uint64_t)q * p + r];
                bounds[(uint64_t)q * (p + 1) + r + 1] = bounds[(uint64_t)q * (p + 1) + r] + v;
                recv[r + 1] += v;
            }
        }
        for (uint32_t r = 0; r < p; ++r) {
            out->recv_counts[r] = recv[r + 1];
            recv[r + 1] += recv[r];
        }
        DSSS_CUDA(cudaMemcpyAsync(L.bounds, bounds.data(), bounds.size() * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(L.recv_begin, recv.data(), (p + 1) * 8, cudaMemcpyHostToDevice, st));
        // (local index, sender PE) of every output position: perm_index in L.dpg, perm_pe in len1
        DSSS_CUDA(cudaMemsetAsync(L.viol, 0, sizeof(uint32_t), st));
        DSSS_TRY(launch_bucket_direct(L.pe, L.g2l, L.bounds, p, p, n, 0, L.lcp, nullptr, nullptr, L.dpg, len1,
                                      out->lcp, L.viol, st));
        pin = (uint32_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin, L.viol, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        if (pin[0]) {
            DSSS_TRY(launch_bucket_direct(L.pe, L.g2l, L.bounds, p, p, n, 0, L.lcp, L.tmp, nullptr, L.dpg, len1,
                                          nullptr, L.viol, st));
            const uint32_t* ins[3] = {L.g2l, L.pe, nullptr};
            uint32_t* outs[3] = {L.dpg, len1, L.out2g};
            DSSS_TRY(multisplit_payload(L.tmp, n, p, 3, ins, outs, nullptr, L.err, L.ms, st));
            DSSS_LAUNCH("k_merged_lcp", st,
                        k_merged_lcp<<<grid_for(n, 256), 256, 0, st>>>(L.out2g, L.lcp, L.recv_begin, p, n, out->lcp));
        }
        DSSS_LAUNCH("k_ms_source", st,
                    k_ms_source<<<grid_for(n, 256), 256, 0, st>>>(out->local_order, L.pb, L.dpg, len1, a, n, source,
                                                                 out->lengths, src_tmp == source ? L.tmp : src_tmp,
                                                                 srcoff));
        len1 = src_tmp == source ? L.tmp : src_tmp;
    }
    // output layout and the strings themselves
    {
        StageTimer t("stage:copy", st);
        DSSS_TRY(exclusive_scan_u32_to_u64(len1, out->offsets, n, (uint64_t*)(total + 1), scan, st));
        pin = (uint32_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin, total + 1, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        const uint64_t bytes = *(const uint64_t*)pin;
        if (bytes > out->chars_capacity)
            return fail(DSSS_EINVAL, "chars_capacity %llu is below the %llu output bytes",
                        (unsigned long long)out->chars_capacity, (unsigned long long)bytes);
        DSSS_TRY(launch_ms_copy(a.chars, srcoff, out->lengths, out->offsets, n, out->chars, st));
    }
    pin = (uint32_t*)ctx->pin;
    DSSS_CUDA(cudaMemcpyAsync(pin, L.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) return fail(DSSS_EDEVICE, "ms sort: internal consistency guard tripped");
    return DSSS_OK;
}

// ----------------------------------------------------------- hQuicksort ----
// RQuick::sort (sorter/RQuick/RQuick.hpp:834-1104, sortRec :415-627) as the
// hQuicksort executable runs it, on one GPU holding every PE.  Strings never
// move between levels: after one global sort, PE q's sorted data at a level is
// the ascending list of global positions it owns (equal strings are
// byte-identical, so which of them a PE holds is immaterial), the exchange
// relabels owners, and the strings are written once at the end: the PEs'
// sorted data in rank order is the global order.  The lists are never built:
// per-tile owner counts, scanned PE-major, give every list's start and the
// rank of every tile in it, so the pivot and each PE's split are a binary
// search over tiles plus a scan of one tile.

constexpr uint32_t HQ_NT = 256, HQ_IPT = 16, HQ_TILE = HQ_NT * HQ_IPT;
constexpr uint32_t HQ_NONE = 0xFFFFFFFFu;

// The pivot's run: lists are searched for the first position of the run of
// strings equal to the pivot and the first position past it.
// glen: lengths in the global order.
__global__ void k_hq_run_ends(const uint32_t* glen, const uint32_t* lcp, uint64_t n, uint32_t* tail) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    tail[g] = g + 1 < n ? !(glen[g] == glen[g + 1] && lcp[g + 1] == glen[g]) : 1u;
}

// Adds owner o of this lane to the shared histogram, one atomic per owner
// and warp (owners come in long runs).
__device__ __forceinline__ void hq_count(uint32_t* h, uint32_t o, uint32_t pw) {
    const uint32_t peers = __match_any_sync(0xffffffffu, o);
    if (o < pw && (threadIdx.x & 31) == (uint32_t)__ffs(peers) - 1) atomicAdd(&h[o], __popc(peers));
}

// The first level's owners: the PE of the string at each global position,
// PEs past the largest power of two pw folded onto PE q - pw (RQuick.hpp:878-959),
// and the owner counts of every tile, PE-major: tc[q * tiles + t].
__global__ void __launch_bounds__(HQ_NT) k_hq_owner0(const uint32_t* ord, uint64_t n, const uint64_t* pb, uint32_t p,
                                                     uint32_t pw, uint64_t tiles, uint16_t* owner, uint32_t* tc) {
    extern __shared__ uint32_t h[];
    for (uint32_t q = threadIdx.x; q < pw; q += HQ_NT) h[q] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * HQ_TILE;
#pragma unroll 4
    for (uint32_t j = 0; j < HQ_IPT; ++j) {
        const uint64_t g = t0 + j * HQ_NT + threadIdx.x;
        uint32_t q = HQ_NONE;
        if (g < n) {
            const uint32_t s = ord[g];
            uint32_t lo = 0, hi = p;  // last q with pb[q] <= s
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(&pb[mid]) <= s) lo = mid;
                else hi = mid;
            }
            q = lo >= pw ? lo - pw : lo;
            owner[g] = (uint16_t)q;
        }
        hq_count(h, q, pw);
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < pw; q += HQ_NT) tc[(uint64_t)q * tiles + blockIdx.x] = h[q];
}

// The exchange (RQuick.hpp:496-586): the left half sends its strings from its
// split on, the right half those before it; dest[q] is q's partner, bit 31 set
// for the left half, cut[q] the position of q's split (HQ_NONE: past its
// end).  The new owners' tile counts are those of the next level.
__global__ void __launch_bounds__(HQ_NT) k_hq_move(uint16_t* owner, uint64_t n, uint32_t pw, uint64_t tiles,
                                                   const uint32_t* cut, const uint32_t* dest, uint32_t* tc) {
    extern __shared__ uint32_t h[];
    for (uint32_t q = threadIdx.x; q < pw; q += HQ_NT) h[q] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * HQ_TILE;
#pragma unroll 4
    for (uint32_t j = 0; j < HQ_IPT; ++j) {
        const uint64_t g = t0 + j * HQ_NT + threadIdx.x;
        uint32_t o = HQ_NONE;
        if (g < n) {
            o = owner[g];
            if (o < pw) {
                const uint32_t c = cut[o], d = dest[o];
                if ((d >> 31) ? (c != HQ_NONE && g >= c) : (c == HQ_NONE || g < c)) {
                    o = d & 0x7FFFFFFFu;
                    owner[g] = (uint16_t)o;
                }
            }
        }
        hq_count(h, o, pw);
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < pw; q += HQ_NT) tc[(uint64_t)q * tiles + blockIdx.x] = h[q];
}

// Strings per PE from the scanned tile counts (off[pw * tiles] is not held:
// the last PE ends at n).
__global__ void k_hq_counts(const uint32_t* off, uint64_t tiles, uint32_t pw, uint64_t n, uint32_t* cnt) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= pw) return;
    const uint64_t e = q + 1 < pw ? off[(uint64_t)(q + 1) * tiles] : n;
    cnt[q] = (uint32_t)(e - off[(uint64_t)q * tiles]);
}

// One level's parameters of PE q, drawn on the host from its random bits.
struct HqPe {
    uint32_t cnt;   // strings q holds
    uint32_t opt;   // locateSplitter's middle: cnt / 2, + 1 by a bit when cnt is odd
    uint32_t piv;   // first PE of a subcube: index of the pivot in its list, HQ_NONE: the empty pivot
    uint32_t cube;  // subcube size at this level
};

__device__ __forceinline__ uint64_t first_not_below(const uint32_t* v, uint64_t m, uint64_t x) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (v[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Block sum and exclusive block scan (HQ_NT threads; sh: HQ_NT / 32 + 1 words).
__device__ __forceinline__ uint32_t hq_block_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    uint32_t pre = x - v, tot = 0;
    for (uint32_t k = 0; k < HQ_NT / 32; ++k) {
        if (k < w) pre += sh[k];
        tot += sh[k];
    }
    __syncthreads();
    total = tot;
    return pre;
}

// Strings of PE q at positions below x (its list's lower bound of x).
__device__ uint32_t hq_rank(const uint16_t* owner, const uint32_t* off, uint64_t tiles, uint64_t n, uint32_t q,
                            uint32_t cnt, uint64_t x, uint32_t* sh) {
    if (x >= n) return cnt;
    const uint64_t t = x / HQ_TILE, t0 = t * HQ_TILE;
    uint32_t c = 0;
    for (uint32_t j = 0; j < HQ_IPT; ++j) {
        const uint64_t g = t0 + j * HQ_NT + threadIdx.x;
        c += g < x && owner[g] == q;
    }
    uint32_t total;
    hq_block_scan(c, sh, total);
    return off[(uint64_t)q * tiles + t] - off[(uint64_t)q * tiles] + total;
}

// Position of the k-th string (from 0, k < its count) of PE q's list.
__device__ uint32_t hq_select(const uint16_t* owner, const uint32_t* off, uint64_t tiles, uint64_t n, uint32_t q,
                              uint32_t k, uint32_t* sh) {
    const uint32_t* row = off + (uint64_t)q * tiles;
    const uint32_t b = row[0];
    uint64_t lo = 0, hi = tiles;  // the last tile whose list rank is <= k
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (row[mid] - b <= k) lo = mid;
        else hi = mid;
    }
    const uint32_t r = k - (row[lo] - b);
    const uint64_t g0 = lo * HQ_TILE + (uint64_t)threadIdx.x * HQ_IPT;
    uint32_t c = 0;
    for (uint32_t j = 0; j < HQ_IPT; ++j) c += g0 + j < n && owner[g0 + j] == q;
    uint32_t total;
    uint32_t pre = hq_block_scan(c, sh, total);
    if (threadIdx.x == 0) sh[HQ_NT / 32] = HQ_NONE;
    __syncthreads();
    if (r >= pre && r < pre + c)
        for (uint32_t j = 0; j < HQ_IPT; ++j)
            if (g0 + j < n && owner[g0 + j] == q) {
                if (pre == r) sh[HQ_NT / 32] = (uint32_t)(g0 + j);
                ++pre;
            }
    __syncthreads();
    const uint32_t v = sh[HQ_NT / 32];
    __syncthreads();
    return v;
}

// locateSplitter (robust, RQuick.hpp:363-385) of PE q = blockIdx.x: the
// subcube's pivot, its run of equal strings, q's lower and upper bound of it,
// the split, and the position where q's split falls.
__global__ void __launch_bounds__(HQ_NT) k_hq_split(const HqPe* prm, const uint16_t* owner, const uint32_t* off,
                                                    uint64_t tiles, const uint32_t* runx, const uint32_t* ord,
                                                    ArenaDev a, uint64_t n, uint32_t pw, uint32_t* cut,
                                                    uint32_t* dest, uint32_t* err) {
    __shared__ uint32_t sh[HQ_NT / 32 + 1];
    const uint32_t q = blockIdx.x;
    const HqPe m = prm[q];
    const uint32_t P = m.cube, b = q & ~(P - 1), half = P >> 1;
    const HqPe r = prm[b];
    uint64_t lo = 0, hi = 0;
    if (r.piv == HQ_NONE) {  // the empty string: every empty string equals it
        uint64_t o;
        uint32_t l;
        str_of(a, ord[0], o, l);
        hi = l == 0 ? first_not_below(runx, n, 1) : 0;
    } else {
        if (r.piv >= r.cnt) {
            if (threadIdx.x == 0) atomicExch(err, 1u);
            return;
        }
        const uint32_t pg = hq_select(owner, off, tiles, n, b, r.piv, sh);
        if (pg >= n) {
            if (threadIdx.x == 0) atomicExch(err, 1u);
            return;
        }
        const uint32_t k = runx[pg];
        lo = first_not_below(runx, n, k);
        hi = first_not_below(runx, n, (uint64_t)k + 1);
    }
    const uint32_t lb = hq_rank(owner, off, tiles, n, q, m.cnt, lo, sh);
    const uint32_t ub = hq_rank(owner, off, tiles, n, q, m.cnt, hi, sh);
    const uint32_t sep = lb < m.opt ? min(m.opt, ub) : lb;
    const uint32_t c = sep < m.cnt ? hq_select(owner, off, tiles, n, q, sep, sh) : HQ_NONE;
    if (threadIdx.x == 0) {
        if (sep < m.cnt && c >= n) atomicExch(err, 1u);
        cut[q] = c;
        dest[q] = (b + (q - b + half) % P) | (q - b < half ? 0x80000000u : 0u);
    }
}

// RandomBitStore (sorter/RQuick/RandomBitStore.hpp:27-52) on PE q's
// std::mt19937_64.
struct HqBits {
    std::mt19937_64 gen;
    uint64_t bits = 0;
    int pos = 64;
    uint32_t next() {
        if (pos == 64) {
            bits = gen();
            pos = 0;
        }
        const uint32_t r = (uint32_t)(bits & 1);
        bits >>= 1;
        ++pos;
        return r;
    }
};

static int hq_sort_dev(Ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* pb, uint64_t seed,
                       dsss_hq_result* out, cudaStream_t st) {
    DSSS_TRY(check_arena(in));
    if (p == 0) return fail(DSSS_EINVAL, "p must be >= 1");
    if (p > MAX_SPLIT_BUCKETS) return fail(DSSS_ENOTSUP, "p > %u PEs per GPU is not supported", MAX_SPLIT_BUCKETS);
    DSSS_TRY(check_parts(p, pb, in->n));
    if (!out || !out->counts || !out->offsets || !out->lengths || (in->n && !out->chars))
        return fail(DSSS_EINVAL, "result arrays missing");
    const uint64_t n = in->n;
    uint32_t pw = 1, levels = 0;
    while (pw * 2 <= p) pw *= 2, ++levels;
    out->levels = levels;
    for (uint32_t q = 0; q < p; ++q) out->counts[q] = 0;
    if (n == 0) return DSSS_OK;
    const uint64_t N = n, tiles = (n + HQ_TILE - 1) / HQ_TILE, cells = tiles * pw;
    if (cells >= (1ull << 32)) return fail(DSSS_ENOTSUP, "hq sort: too many tiles x PEs");
    const uint32_t smax = 0;
    auto plan = [&](Carve& c, ulonglong2*& handles, uint32_t*& ord, uint32_t*& lcp, uint16_t*& owner, uint32_t*& tmp,
                    uint32_t*& runx, uint32_t*& srcb, uint32_t*& tc, uint32_t*& off, uint32_t*& cnt, HqPe*& prm,
                    uint32_t*& cut, uint32_t*& dest, uint32_t*& err, uint64_t*& pbd, uint64_t*& total, void*& scan,
                    uint64_t*& srcoff, SortLayout& sl) {
        handles = c.take<ulonglong2>(N);
        ord = c.take<uint32_t>(N);
        lcp = c.take<uint32_t>(N);
        owner = c.take<uint16_t>(N);
        tmp = c.take<uint32_t>(N);
        runx = c.take<uint32_t>(N);
        srcb = out->source ? nullptr : c.take<uint32_t>(N);
        srcoff = c.take<uint64_t>(N);
        tc = c.take<uint32_t>(cells);
        off = c.take<uint32_t>(cells);
        cnt = c.take<uint32_t>(MAX_SPLIT_BUCKETS);
        prm = c.take<HqPe>(MAX_SPLIT_BUCKETS);
        cut = c.take<uint32_t>(MAX_SPLIT_BUCKETS);
        dest = c.take<uint32_t>(MAX_SPLIT_BUCKETS);
        err = c.take<uint32_t>(1);
        pbd = c.take<uint64_t>(p + 1);
        total = c.take<uint64_t>(2);
        scan = c.take<unsigned char>(scan_scratch_bytes(N > cells ? N : cells));
        layout_sort(c, sl, N, 1, smax);
    };
    ulonglong2* handles;
    uint32_t *ord, *lcp, *tmp, *runx, *srcb, *tc, *off, *cnt, *cut, *dest, *err;
    uint16_t* owner;
    HqPe* prm;
    uint64_t *pbd, *total, *srcoff;
    void* scan;
    SortLayout sl;
    Carve sz(nullptr);
    plan(sz, handles, ord, lcp, owner, tmp, runx, srcb, tc, off, cnt, prm, cut, dest, err, pbd, total, scan, srcoff, sl);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    const uint64_t pin_bytes = MAX_SPLIT_BUCKETS * (sizeof(uint32_t) + sizeof(HqPe)) + 64;
    DSSS_TRY(ensure_pin(ctx, pin_bytes < 4096 ? 4096 : pin_bytes));
    Carve c(ctx->ws);
    plan(c, handles, ord, lcp, owner, tmp, runx, srcb, tc, off, cnt, prm, cut, dest, err, pbd, total, scan, srcoff, sl);
    ArenaDev a = view(in);
    make_handles(a, handles, st);
    a.h = handles;
    DSSS_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
    const uint64_t set_begin[2] = {0, n};
    {
        StageTimer t("stage:sort", st);
        DSSS_TRY(sort_strings(sl, a, n, 1, set_begin, nullptr, ord, lcp, smax, (uint32_t*)ctx->pin, st));
    }
    // the output layout: the PEs' sorted data in rank order is the global order
    uint32_t* source = out->source ? out->source : srcb;
    {
        StageTimer t("stage:layout", st);
        DSSS_LAUNCH("k_ms_source", st,
                    k_ms_source<<<grid_for(n, 256), 256, 0, st>>>(ord, nullptr, nullptr, nullptr, a, n, source,
                                                                 out->lengths, tmp, srcoff));
        DSSS_TRY(exclusive_scan_u32_to_u64(tmp, out->offsets, n, total, scan, st));
        DSSS_CUDA(cudaMemcpyAsync(ctx->pin, total, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        const uint64_t bytes = *(const uint64_t*)ctx->pin;
        if (bytes > out->chars_capacity)
            return fail(DSSS_EINVAL, "chars_capacity %llu is below the %llu output bytes",
                        (unsigned long long)out->chars_capacity, (unsigned long long)bytes);
    }
    if (levels == 0) {  // one PE: the local sort is the result (RQuick.hpp:855-864)
        out->counts[0] = n;
    } else {
        StageTimer t("stage:levels", st);
        DSSS_CUDA(cudaMemcpyAsync(pbd, pb, (p + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_hq_run_ends", st,
                    k_hq_run_ends<<<grid_for(n, 256), 256, 0, st>>>(out->lengths, lcp, n, tmp));
        DSSS_TRY(exclusive_scan_u32(tmp, runx, n, nullptr, scan, st));
        const size_t hsm = pw * sizeof(uint32_t);
        DSSS_LAUNCH("k_hq_owner0", st,
                    k_hq_owner0<<<(unsigned)tiles, HQ_NT, hsm, st>>>(ord, n, pbd, p, pw, tiles, owner, tc));
        std::vector<HqBits> bits(pw);
        for (uint32_t q = 0; q < pw; ++q) bits[q].gen.seed(seed + q);  // HQuicksort.cpp:344-345
        uint32_t* hcnt = (uint32_t*)ctx->pin;
        HqPe* hprm = (HqPe*)((char*)ctx->pin + MAX_SPLIT_BUCKETS * sizeof(uint32_t));
        for (uint32_t P = pw;; P >>= 1) {
            DSSS_TRY(exclusive_scan_u32(tc, off, cells, nullptr, scan, st));
            DSSS_LAUNCH("k_hq_counts", st, k_hq_counts<<<grid_for(pw, 128), 128, 0, st>>>(off, tiles, pw, n, cnt));
            DSSS_CUDA(cudaMemcpyAsync(hcnt, cnt, pw * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaStreamSynchronize(st));
            if (P < 2) break;  // the counts after the last level
            // the bits in the reference's order per PE: middleMostElements
            // (:273-314), the first PE's selectMedian
            // (BinTreeMedianSelection.hpp:135-152), locateSplitter (:363-385)
            uint64_t sum = 0;
            for (uint32_t q = 0; q < pw; ++q) {
                const uint32_t k = hcnt[q];
                HqPe& m = hprm[q];
                sum += k;
                m.cnt = k;
                m.cube = P;
                m.piv = HQ_NONE;
                const uint32_t beg = k > 2 ? (k - 2) / 2 + (k % 2 == 1 ? bits[q].next() : 0u) : 0u;
                if (q % P == 0) {
                    const uint32_t nm = k < 2 ? k : 2;
                    if (nm) m.piv = beg + (nm == 2 ? bits[q].next() : 0u);
                }
                m.opt = k / 2 + (k % 2 == 1 ? bits[q].next() : 0u);
            }
            if (sum != n) return fail(DSSS_EDEVICE, "hq sort: owner counts add up to %llu, not %llu",
                                      (unsigned long long)sum, (unsigned long long)n);
            DSSS_CUDA(cudaMemcpyAsync(prm, hprm, pw * sizeof(HqPe), cudaMemcpyHostToDevice, st));
            DSSS_LAUNCH("k_hq_split", st,
                        k_hq_split<<<pw, HQ_NT, 0, st>>>(prm, owner, off, tiles, runx, ord, a, n, pw, cut, dest, err));
            DSSS_LAUNCH("k_hq_move", st,
                        k_hq_move<<<(unsigned)tiles, HQ_NT, hsm, st>>>(owner, n, pw, tiles, cut, dest, tc));
            // the pinned parameters are rewritten only after the next count
            // read-back, which the stream orders after this copy
        }
        uint64_t sum = 0;
        for (uint32_t q = 0; q < pw; ++q) sum += out->counts[q] = hcnt[q];
        if (sum != n) return fail(DSSS_EDEVICE, "hq sort: final counts add up to %llu, not %llu",
                                  (unsigned long long)sum, (unsigned long long)n);
    }
    {
        StageTimer t("stage:copy", st);
        DSSS_TRY(launch_ms_copy(a.chars, srcoff, out->lengths, out->offsets, n, out->chars, st));
    }
    DSSS_CUDA(cudaMemcpyAsync(ctx->pin, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (*(const uint32_t*)ctx->pin) return fail(DSSS_EDEVICE, "hq sort: internal consistency guard tripped");
    return DSSS_OK;
}

}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_hq_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin, uint64_t seed,
                 dsss_hq_result* out, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return hq_sort_dev(ctx, in, p, part_begin, seed, out, (cudaStream_t)stream);
}

int dsss_ms_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin, const dsss_opts* opts,
                 dsss_ms_result* out, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return ms_sort_dev(ctx, in, p, part_begin, opts, out, (cudaStream_t)stream);
}

int dsss_pd_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin, const dsss_opts* opts,
                 dsss_pd_result* out, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return pd_sort_dev(ctx, in, 1, p, part_begin, opts, out, (cudaStream_t)stream);
}

int dsss_pd_sort_batched(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p, const uint64_t* part_begin,
                         const dsss_opts* opts, dsss_pd_result* out, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return pd_sort_dev(ctx, in, nsets, p, part_begin, opts, out, (cudaStream_t)stream);
}

int dsss_local_sort_lcp(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                        const dsss_opts* opts, uint32_t* order, uint32_t* lcp, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    DSSS_TRY(check_parts(p, part_begin, in->n));
    if (in->n && (!order || !lcp)) return fail(DSSS_EINVAL, "order/lcp is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t smax = smallmax_of(opts);
    Carve sz(nullptr);
    SortLayout L;
    sz.take<ulonglong2>(in->n ? in->n : 1);
    layout_sort(sz, L, in->n, p, smax);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    ulonglong2* h = c.take<ulonglong2>(in->n ? in->n : 1);
    layout_sort(c, L, in->n, p, smax);
    ArenaDev a = view(in);
    make_handles(a, h, st);
    a.h = h;
    return sort_strings(L, a, in->n, p, part_begin, nullptr, order, lcp, smax, (uint32_t*)ctx->pin, st);
}

int dsss_dp_prefixes(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                     const uint32_t* order, const uint32_t* lcp, uint32_t* dp, uint64_t* round_counts,
                     uint32_t max_rounds, uint32_t* rounds, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    DSSS_TRY(check_parts(p, part_begin, in->n));
    if (in->n && (!order || !lcp || !dp)) return fail(DSSS_EINVAL, "order/lcp/dp is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    DpLayout L;
    sz.take<ulonglong2>(in->n ? in->n : 1);
    layout_dp(sz, L, in->n);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    ulonglong2* h = c.take<ulonglong2>(in->n ? in->n : 1);
    layout_dp(c, L, in->n);
    ArenaDev a = view(in);
    make_handles(a, h, (cudaStream_t)stream);
    a.h = h;
    // The PE split needs no extra handling: every PE's first LCP is 0, so no
    // string is an LCP duplicate of the previous PE's last one.
    return dp_rounds(L, a, in->n, order, lcp, dp, round_counts, max_rounds, rounds, (uint32_t*)ctx->pin,
                     (cudaStream_t)stream);
}

int dsss_dp_round(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, const uint32_t* lcp,
                  const uint32_t* candidates, uint64_t m, uint32_t depth, uint32_t* results, uint32_t* next,
                  uint64_t* m_next, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    if (!m_next) return fail(DSSS_EINVAL, "m_next is NULL");
    if (in->n && (!order || !lcp || !results || !next)) return fail(DSSS_EINVAL, "order/lcp/results/next is NULL");
    if (candidates && m > in->n) return fail(DSSS_EINVAL, "more candidates than strings");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    DpRoundLayout R;
    layout_dp_round(sz, R, in->n);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_dp_round(c, R, in->n);
    return dp_one_round(R, view(in), in->n, order, lcp, candidates, m, depth, results, next, m_next,
                        (uint32_t*)ctx->pin, (cudaStream_t)stream);
}

int dsss_bucket_scatter(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                        const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, const uint64_t* intervals,
                        uint8_t* recv_chars, uint64_t recv_capacity, uint64_t* char_total, uint64_t* recv_char_begin,
                        uint32_t* recv_char_start, uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe,
                        uint64_t* recv_counts, uint64_t* recv_offsets, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    DSSS_TRY(check_parts(p, part_begin, in->n));
    if (!intervals || !char_total) return fail(DSSS_EINVAL, "intervals/char_total is NULL");
    if (in->n && (!local_order || !lcp || !dp || !recv_lcp || !recv_index || !recv_pe))
        return fail(DSSS_EINVAL, "input or per-string output array is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    Carve sz(nullptr);
    ExchangeLayout L;
    layout_exchange(sz, L, in->n, p);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    layout_exchange(c, L, in->n, p);
    DSSS_TRY(bucket_scatter(L, view(in), p, part_begin, local_order, lcp, dp, intervals, char_total, recv_chars,
                            recv_capacity, recv_char_begin, recv_lcp, recv_index, recv_pe, recv_counts, recv_offsets,
                            (uint32_t*)ctx->pin, st));
    if (recv_char_start && in->n)
        DSSS_CUDA(cudaMemcpyAsync(recv_char_start, L.cstart, in->n * 4, cudaMemcpyDeviceToDevice, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

int dsss_lcp_merge(dsss_ctx* ctx, const uint8_t* recv_chars, uint64_t char_bytes, const uint32_t* recv_char_start,
                   const uint32_t* recv_lcp, uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* recv_counts,
                   const uint64_t* recv_offsets, uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp,
                   uint32_t* perm_index, uint32_t* perm_pe, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (nrecv == 0 || p == 0 || !recv_counts) return fail(DSSS_EINVAL, "nrecv/p/recv_counts missing");
    if (n && (!recv_chars || !recv_lcp || !order)) return fail(DSSS_EINVAL, "recv_chars/recv_lcp/order is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    int rc = lcp_merge(ctx, recv_chars, char_bytes, recv_char_start, recv_lcp, n, nrecv, p, recv_counts, recv_offsets,
                       order, merged_lcp, old_lcp, perm_index, perm_pe, (cudaStream_t)stream);
    return rc;
}

int dsss_lcp_merge_strings(dsss_ctx* ctx, const uint8_t* recv_chars, uint64_t char_bytes,
                           const uint32_t* recv_char_start, const uint32_t* recv_lcp, uint64_t n, uint32_t nrecv,
                           uint32_t p, const uint64_t* recv_counts, const uint64_t* recv_offsets, uint32_t* order,
                           uint32_t* merged_lcp, uint8_t* out_chars, uint64_t out_capacity, uint64_t* out_offsets,
                           uint32_t* out_lengths, uint64_t* out_bytes, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (nrecv == 0 || p == 0 || !recv_counts || !out_bytes) return fail(DSSS_EINVAL, "nrecv/p/recv_counts/out_bytes missing");
    if (n && (!recv_chars || !recv_lcp || !order || !out_chars || !out_offsets || !out_lengths))
        return fail(DSSS_EINVAL, "input or output arrays are NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    return lcp_merge_strings(ctx, recv_chars, char_bytes, recv_char_start, recv_lcp, n, nrecv, p, recv_counts,
                             recv_offsets, order, merged_lcp, nullptr, nullptr, nullptr, out_chars, out_capacity,
                             out_offsets, out_lengths, out_bytes, (cudaStream_t)stream);
}

int dsss_prefix_hash(const dsss_arena* in, const uint32_t* ids, uint64_t m, uint32_t depth, uint64_t* hash,
                     dsss_stream_t stream) {
    DSSS_TRY(check_arena(in));
    if (m && (!ids || !hash)) return fail(DSSS_EINVAL, "ids/hash is NULL");
    return prefix_hash(view(in), ids, m, depth, hash, (cudaStream_t)stream);
}

int dsss_partition(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                   const uint32_t* order, const uint32_t* dp, const dsss_opts* opts, uint64_t* intervals,
                   dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    DSSS_TRY(check_parts(p, part_begin, in->n));
    if (!intervals || (in->n && (!order || !dp))) return fail(DSSS_EINVAL, "order/dp/intervals is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    const uint32_t factor = factor_of(opts);
    Carve sz(nullptr);
    PartitionLayout L;
    layout_partition(sz, L, in->n, p, factor);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    Carve c(ctx->ws);
    layout_partition(c, L, in->n, p, factor);
    return partition_pes(L, ctx, view(in), p, part_begin, order, dp, sampler_of(opts), factor, intervals,
                         (cudaStream_t)stream);
}

int dsss_adjacent_lcp(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, uint64_t m, uint32_t* lcp,
                      dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    DSSS_TRY(check_arena(in));
    if (m && (!order || !lcp)) return fail(DSSS_EINVAL, "order/lcp is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    Carve sz(nullptr);
    sz.take<uint32_t>(m + 1);
    sz.take<uint32_t>(1);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    Carve c(ctx->ws);
    uint32_t* longq = c.take<uint32_t>(m + 1);
    uint32_t* nlong = c.take<uint32_t>(1);
    return adjacent_lcp(view(in), order, m, lcp, longq, nlong, (cudaStream_t)stream);
}

// Host-memory variant: device copies of the arena and results live in a
// second context buffer so repeated calls reuse it.
static int pd_sort_host(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p, const uint64_t* part_begin,
                        const dsss_opts* opts, dsss_pd_result* out, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (!in) return fail(DSSS_EINVAL, "arena is NULL");
    if (nsets == 0 || p == 0) return fail(DSSS_EINVAL, "nsets and p must be >= 1");
    DSSS_TRY(check_parts(nsets * p, part_begin, in->n));
    if (!out) return fail(DSSS_EINVAL, "result is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t n = in->n;
    const bool llcp = opts && (opts->flags & DSSS_FLAG_LOCAL_LCP) && out->local_lcp;
    auto plan = [&](Carve& c, dsss_arena& da, dsss_pd_result& dr) {
        uint8_t* chars = c.take<uint8_t>(in->char_bytes + 64);
        uint64_t* off = c.take<uint64_t>(n ? n : 1);
        uint32_t* len = c.take<uint32_t>(n ? n : 1);
        da = dsss_arena{chars, in->char_bytes, off, len, n};
        dr = *out;
        dr.local_order = c.take<uint32_t>(n ? n : 1);
        dr.local_lcp = llcp ? c.take<uint32_t>(n ? n : 1) : nullptr;
        dr.dp = c.take<uint32_t>(n ? n : 1);
        dr.perm_index = c.take<uint32_t>(n ? n : 1);
        dr.perm_pe = c.take<uint32_t>(n ? n : 1);
        dr.merged_lcp = out->merged_lcp ? c.take<uint32_t>(n ? n : 1) : nullptr;
    };
    Carve sz(nullptr);
    dsss_arena da;
    dsss_pd_result dr;
    plan(sz, da, dr);
    // The io buffer sits in front of the pipeline's own scratch.
    Carve pdsz(nullptr);
    PdLayout PL;
    layout_pd(pdsz, PL, n, nsets, p, factor_of(opts), smallmax_of(opts));
    const uint64_t io_bytes = (sz.used + 255) & ~255ull;
    DSSS_TRY(ensure_ws(ctx, io_bytes + pdsz.used));
    Carve c(ctx->ws);
    plan(c, da, dr);
    if (in->char_bytes) DSSS_CUDA(cudaMemcpyAsync((void*)da.chars, in->chars, in->char_bytes, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemsetAsync((uint8_t*)da.chars + in->char_bytes, 0, 64, st));
    if (n) {
        DSSS_CUDA(cudaMemcpyAsync((void*)da.offsets, in->offsets, n * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync((void*)da.lengths, in->lengths, n * 4, cudaMemcpyHostToDevice, st));
    }
    // Run the device path on the scratch behind the io block.
    Ctx sub = *ctx;
    sub.ws = (char*)ctx->ws + io_bytes;
    sub.ws_cap = ctx->ws_cap - io_bytes;
    sub.fixed_ws = true;
    int rc = pd_sort_dev(&sub, &da, nsets, p, part_begin, opts, &dr, st);
    ctx->pin = sub.pin;
    ctx->pin_cap = sub.pin_cap;
    if (rc != DSSS_OK) return rc;
    if (n) {
        DSSS_CUDA(cudaMemcpyAsync(out->local_order, dr.local_order, n * 4, cudaMemcpyDeviceToHost, st));
        if (llcp) DSSS_CUDA(cudaMemcpyAsync(out->local_lcp, dr.local_lcp, n * 4, cudaMemcpyDeviceToHost, st));
        if (p > 1) {
            DSSS_CUDA(cudaMemcpyAsync(out->dp, dr.dp, n * 4, cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaMemcpyAsync(out->perm_index, dr.perm_index, n * 4, cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaMemcpyAsync(out->perm_pe, dr.perm_pe, n * 4, cudaMemcpyDeviceToHost, st));
            if (out->merged_lcp)
                DSSS_CUDA(cudaMemcpyAsync(out->merged_lcp, dr.merged_lcp, n * 4, cudaMemcpyDeviceToHost, st));
        }
    }
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

int dsss_pd_sort_host(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                      const dsss_opts* opts, dsss_pd_result* out, dsss_stream_t stream) {
    return pd_sort_host(ctx, in, 1, p, part_begin, opts, out, stream);
}

int dsss_pd_sort_batched_host(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p,
                              const uint64_t* part_begin, const dsss_opts* opts, dsss_pd_result* out,
                              dsss_stream_t stream) {
    return pd_sort_host(ctx, in, nsets, p, part_begin, opts, out, stream);
}

}  // extern "C"
