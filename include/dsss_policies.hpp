// dsss_policies.hpp — C++ host adaptors over the C ABI (dsss.h) that present
// the reference's prefix-doubling interfaces, so code written against
// bingmann/distributed-string-sorting can call the B200 path with its own
// data layout: NUL-terminated strings back to back per PE (the raw vector of
// StringLcpContainer, src/strings/stringcontainer.hpp:163-433), size_t
// indices and LCPs, and the StringIndexPEIndex permutation (util/structs.hpp).
//
// One GPU holds all p PEs, so each adaptor takes every PE's strings at once
// where the reference runs one call per MPI rank.  Errors throw dsss_gpu::Error
// (the reference aborts).  Link with -ldsss (libdsss.so) and the CUDA runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "dsss.h"

namespace dsss_gpu {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != DSSS_OK) throw Error(rc, dsss_last_error());
}

inline void check_cuda(cudaError_t e) {
    if (e != cudaSuccess) throw Error(DSSS_EDEVICE, cudaGetErrorString(e));
}

// Owns a dsss_ctx (reusable device scratch).  One per host thread.
class Context {
public:
    explicit Context(int device = 0, uint64_t hbm_budget = 0) { check(dsss_ctx_create(device, hbm_budget, &h_)); }
    ~Context() { dsss_ctx_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    dsss_ctx* get() const { return h_; }

private:
    dsss_ctx* h_ = nullptr;
};

// util/structs.hpp: the PD path's output element.
struct StringIndexPEIndex {
    size_t stringIndex;
    size_t PEIndex;
};

// Sampling policies of computePartition (samplingStrategies.hpp).
enum class Sampler : uint32_t { NumStrings = DSSS_SAMPLER_NUM_STRINGS, IndexedNumStrings = DSSS_SAMPLER_INDEXED_NUM_STRINGS };

// Host string arena built from per-PE raw vectors (NUL-terminated strings).
struct HostArena {
    std::vector<uint8_t> chars;
    std::vector<uint64_t> offsets;
    std::vector<uint32_t> lengths;
    std::vector<uint64_t> part_begin;

    explicit HostArena(const std::vector<std::vector<unsigned char>>& raw_per_pe) {
        size_t total = 0;
        for (auto& r : raw_per_pe) total += r.size();
        chars.reserve(total + 64);
        part_begin.push_back(0);
        for (auto& r : raw_per_pe) {
            size_t i = 0;
            while (i < r.size()) {
                size_t j = i;
                while (j < r.size() && r[j] != 0) ++j;
                if (j == r.size()) throw Error(DSSS_EINVAL, "raw strings must end with a NUL");
                offsets.push_back(chars.size() + i);
                lengths.push_back(static_cast<uint32_t>(j - i));
                i = j + 1;
            }
            chars.insert(chars.end(), r.begin(), r.end());
            part_begin.push_back(offsets.size());
        }
        chars.resize(chars.size() + 64, 0);  // padding the device copy relies on
    }
    size_t n() const { return offsets.size(); }
    uint32_t p() const { return static_cast<uint32_t>(part_begin.size() - 1); }
    dsss_arena view() const {
        return dsss_arena{chars.data(), chars.size() - 64, offsets.data(), lengths.data(), offsets.size()};
    }
};

// Device copy of a HostArena (RAII).
struct DeviceArena {
    uint8_t* chars = nullptr;
    uint64_t* offsets = nullptr;
    uint32_t* lengths = nullptr;
    uint64_t char_bytes = 0, n = 0;
    explicit DeviceArena(const HostArena& h) : char_bytes(h.chars.size() - 64), n(h.n()) {
        check_cuda(cudaMalloc(&chars, h.chars.size()));
        check_cuda(cudaMalloc(&offsets, (n ? n : 1) * 8));
        check_cuda(cudaMalloc(&lengths, (n ? n : 1) * 4));
        check_cuda(cudaMemcpy(chars, h.chars.data(), h.chars.size(), cudaMemcpyHostToDevice));
        if (n) {
            check_cuda(cudaMemcpy(offsets, h.offsets.data(), n * 8, cudaMemcpyHostToDevice));
            check_cuda(cudaMemcpy(lengths, h.lengths.data(), n * 4, cudaMemcpyHostToDevice));
        }
    }
    ~DeviceArena() {
        cudaFree(chars);
        cudaFree(offsets);
        cudaFree(lengths);
    }
    DeviceArena(const DeviceArena&) = delete;
    DeviceArena& operator=(const DeviceArena&) = delete;
    dsss_arena view() const { return dsss_arena{chars, char_bytes, offsets, lengths, n}; }
};

template <typename T>
struct DeviceVec {
    T* p = nullptr;
    size_t n = 0;
    explicit DeviceVec(size_t count) : n(count) { check_cuda(cudaMalloc(&p, (count ? count : 1) * sizeof(T))); }
    DeviceVec(const std::vector<T>& h) : DeviceVec(h.size()) {
        if (n) check_cuda(cudaMemcpy(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    }
    ~DeviceVec() { cudaFree(p); }
    DeviceVec(const DeviceVec&) = delete;
    std::vector<T> host() const {
        std::vector<T> h(n);
        if (n) check_cuda(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
        return h;
    }
};

template <typename A, typename B>
inline std::vector<A> widen(const std::vector<B>& v) {
    return std::vector<A>(v.begin(), v.end());
}

// Results of DistributedPrefixDoublingSort::sort for every PE.
struct PdSortResult {
    // Per PE: input position (within that PE's raw vector) of each locally
    // sorted string — the order radixsort_CI3 leaves the PE's container in.
    std::vector<std::vector<size_t>> local_order;
    std::vector<std::vector<size_t>> dp;                   // per PE, local order
    std::vector<std::vector<size_t>> interval_sizes;       // per PE: strings sent to each PE
    std::vector<std::vector<StringIndexPEIndex>> permutation;  // per receiving PE
    std::vector<std::vector<size_t>> merged_lcp;           // per receiving PE
};

// DistributedPrefixDoublingSort<StringLcpPtr, Sampler, AllToAllStringImplPrefixDoubling,
// AllToAllHashesNaive>::sort (src/sorter/distributed/prefix_doubling.hpp:200-295)
// for all PEs at once.  As in the reference, p == 1 returns after the local
// sort with an empty permutation (:236).
class DistributedPrefixDoublingSort {
public:
    explicit DistributedPrefixDoublingSort(Sampler s = Sampler::NumStrings) : sampler_(s) {}

    PdSortResult sort(Context& ctx, const std::vector<std::vector<unsigned char>>& raw_per_pe,
                      cudaStream_t stream = nullptr) const {
        HostArena h(raw_per_pe);
        const size_t n = h.n();
        const uint32_t p = h.p();
        std::vector<uint32_t> order(n ? n : 1), dp(n ? n : 1), pidx(n ? n : 1), ppe(n ? n : 1), mlcp(n ? n : 1);
        std::vector<uint64_t> intervals((size_t)p * p), recv(p);
        dsss_pd_result r{order.data(), nullptr, dp.data(), intervals.data(), pidx.data(), ppe.data(), mlcp.data(),
                         recv.data()};
        dsss_opts o{static_cast<uint32_t>(sampler_), 2, 0, 0};
        dsss_arena a = h.view();
        check(dsss_pd_sort_host(ctx.get(), &a, p, h.part_begin.data(), &o, &r, (dsss_stream_t)stream));
        PdSortResult out;
        out.local_order.resize(p);
        out.dp.resize(p);
        out.interval_sizes.resize(p);
        for (uint32_t q = 0; q < p; ++q) {
            for (uint64_t i = h.part_begin[q]; i < h.part_begin[q + 1]; ++i) {
                out.local_order[q].push_back(order[i] - h.part_begin[q]);
                if (p > 1) out.dp[q].push_back(dp[i]);
            }
            if (p > 1)
                out.interval_sizes[q].assign(intervals.begin() + (size_t)q * p, intervals.begin() + (size_t)(q + 1) * p);
        }
        out.permutation.resize(p);
        out.merged_lcp.resize(p);
        size_t k = 0;
        for (uint32_t r2 = 0; r2 < p; ++r2)
            for (uint64_t j = 0; j < recv[r2]; ++j, ++k) {
                out.permutation[r2].push_back({pidx[k], ppe[k]});
                out.merged_lcp[r2].push_back(mlcp[k]);
            }
        return out;
    }

private:
    Sampler sampler_;
};

// Results of DistributedMergeSort::sort for every PE.
struct MsSortResult {
    std::vector<std::vector<size_t>> local_order;     // per PE, as in PdSortResult
    std::vector<std::vector<size_t>> interval_sizes;  // per PE: strings sent to each PE
    // Per receiving PE: the returned StringLcpContainer's raw strings
    // (NUL-terminated, in order) and LCPs (0 first).
    std::vector<std::vector<unsigned char>> raw_strings;
    std::vector<std::vector<size_t>> lcps;
    size_t avg_lcp = 0;  // getAvgLcp over all PEs
};

// DistributedMergeSort<StringLcpPtr, SampleSplittersNumStringsPolicy,
// AllToAllStringImpl<..., EmptyLcpByteEncoderMemCpy>, ...>::sort
// (src/sorter/distributed/lcp_aware_number_string_splitting.hpp:184-290) for
// all PEs at once.  As in the reference, p == 1 returns the local sort.
class DistributedMergeSort {
public:
    MsSortResult sort(Context& ctx, const std::vector<std::vector<unsigned char>>& raw_per_pe,
                      cudaStream_t stream = nullptr) const {
        HostArena h(raw_per_pe);
        DeviceArena d(h);
        const size_t n = h.n();
        const uint32_t p = h.p();
        const uint64_t cap = h.chars.size() - 64;  // every string and its NUL
        DeviceVec<uint32_t> order(n), lens(n), lcp(n);
        DeviceVec<uint64_t> offs(n);
        DeviceVec<uint8_t> chars(cap + 64);
        std::vector<uint64_t> intervals((size_t)p * p), recv(p);
        dsss_ms_result r{order.p, intervals.data(), chars.p, cap, offs.p, lens.p, lcp.p, nullptr, recv.data(), 0};
        dsss_opts o{DSSS_SAMPLER_NUM_STRINGS, 2, 0, 0};
        dsss_arena a = d.view();
        check(dsss_ms_sort(ctx.get(), &a, p, h.part_begin.data(), &o, &r, (dsss_stream_t)stream));
        check_cuda(cudaStreamSynchronize(stream));
        const std::vector<uint32_t> ho = order.host(), hl = lcp.host();
        const std::vector<uint8_t> hc = chars.host();
        MsSortResult out;
        out.avg_lcp = r.avg_lcp;
        out.local_order.resize(p);
        out.interval_sizes.resize(p);
        for (uint32_t q = 0; q < p; ++q) {
            for (uint64_t i = h.part_begin[q]; i < h.part_begin[q + 1]; ++i)
                out.local_order[q].push_back(ho[i] - h.part_begin[q]);
            out.interval_sizes[q].assign(intervals.begin() + (size_t)q * p, intervals.begin() + (size_t)(q + 1) * p);
        }
        out.raw_strings.resize(p);
        out.lcps.resize(p);
        size_t k = 0, byte = 0;
        for (uint32_t q = 0; q < p; ++q)
            for (uint64_t j = 0; j < recv[q]; ++j, ++k) {
                size_t e = byte;
                while (hc[e] != 0) ++e;
                out.raw_strings[q].insert(out.raw_strings[q].end(), hc.begin() + byte, hc.begin() + e + 1);
                out.lcps[q].push_back(hl[k]);
                byte = e + 1;
            }
        return out;
    }
};

// RQuick::sort(generator, std::move(data), MPI_BYTE, tag, comm,
// StringComparator(), true) (src/sorter/RQuick/RQuick.hpp:1109-1115) as the
// hQuicksort executable calls it (src/executables/HQuicksort.cpp:344-356,
// PE r's generator seeded with 3469931 + r) for all PEs at once: every PE's
// returned container as raw NUL-terminated strings in sorted order.
class RQuick {
public:
    explicit RQuick(uint64_t seed = 3469931) : seed_(seed) {}
    std::vector<std::vector<unsigned char>> sort(Context& ctx,
                                                 const std::vector<std::vector<unsigned char>>& raw_per_pe,
                                                 cudaStream_t stream = nullptr) const {
        HostArena h(raw_per_pe);
        DeviceArena d(h);
        const size_t n = h.n();
        const uint32_t p = h.p();
        const uint64_t cap = h.chars.size() - 64;  // every string and its NUL
        DeviceVec<uint32_t> lens(n);
        DeviceVec<uint64_t> offs(n);
        DeviceVec<uint8_t> chars(cap + 64);
        std::vector<uint64_t> counts(p);
        dsss_hq_result r{counts.data(), chars.p, cap, offs.p, lens.p, nullptr, 0};
        dsss_arena a = d.view();
        check(dsss_hq_sort(ctx.get(), &a, p, h.part_begin.data(), seed_, &r, (dsss_stream_t)stream));
        check_cuda(cudaStreamSynchronize(stream));
        const std::vector<uint8_t> hc = chars.host();
        std::vector<std::vector<unsigned char>> out(p);
        size_t byte = 0;
        for (uint32_t q = 0; q < p; ++q)
            for (uint64_t j = 0; j < counts[q]; ++j) {
                size_t e = byte;
                while (hc[e] != 0) ++e;
                out[q].insert(out[q].end(), hc.begin() + byte, hc.begin() + e + 1);
                byte = e + 1;
            }
        return out;
    }

private:
    uint64_t seed_;
};

// tlx::sort_strings_detail::radixsort_CI3(StringLcpPtr, 0, 0) for each PE:
// order[q][i] = input position of the i-th smallest string of PE q,
// lcp[q][i] = LCP with its predecessor (0 first).
inline void radixsort_CI3(Context& ctx, const std::vector<std::vector<unsigned char>>& raw_per_pe,
                          std::vector<std::vector<size_t>>& order, std::vector<std::vector<size_t>>& lcp) {
    HostArena h(raw_per_pe);
    DeviceArena d(h);
    DeviceVec<uint32_t> o(h.n()), l(h.n());
    dsss_arena a = d.view();
    check(dsss_local_sort_lcp(ctx.get(), &a, h.p(), h.part_begin.data(), nullptr, o.p, l.p, nullptr));
    check_cuda(cudaDeviceSynchronize());
    auto ho = o.host(), hl = l.host();
    order.assign(h.p(), {});
    lcp.assign(h.p(), {});
    for (uint32_t q = 0; q < h.p(); ++q)
        for (uint64_t i = h.part_begin[q]; i < h.part_begin[q + 1]; ++i) {
            order[q].push_back(ho[i] - h.part_begin[q]);
            lcp[q].push_back(hl[i]);
        }
}

// computeDistinguishingPrefixes (prefix_doubling.hpp:156-198) for every PE,
// on strings already in local order (as radixsort_CI3 leaves them): results
// per PE in that order, plus the candidate count after each round.
inline std::vector<std::vector<size_t>> computeDistinguishingPrefixes(
    Context& ctx, const std::vector<std::vector<unsigned char>>& sorted_raw_per_pe,
    const std::vector<std::vector<size_t>>& lcp_per_pe, std::vector<uint64_t>* round_counts = nullptr) {
    HostArena h(sorted_raw_per_pe);
    DeviceArena d(h);
    std::vector<uint32_t> ord(h.n()), l;
    for (size_t i = 0; i < h.n(); ++i) ord[i] = static_cast<uint32_t>(i);
    for (auto& v : lcp_per_pe)
        for (size_t x : v) l.push_back(static_cast<uint32_t>(x));
    if (l.size() != h.n()) throw Error(DSSS_EINVAL, "one LCP per string expected");
    DeviceVec<uint32_t> dord(ord), dl(l), ddp(h.n());
    std::vector<uint64_t> counts(64);
    uint32_t rounds = 0;
    dsss_arena a = d.view();
    check(dsss_dp_prefixes(ctx.get(), &a, h.p(), h.part_begin.data(), dord.p, dl.p, ddp.p, counts.data(), 64, &rounds,
                           nullptr));
    check_cuda(cudaDeviceSynchronize());
    if (round_counts) round_counts->assign(counts.begin(), counts.begin() + (rounds < 64 ? rounds : 64));
    auto hdp = ddp.host();
    std::vector<std::vector<size_t>> out(h.p());
    for (uint32_t q = 0; q < h.p(); ++q)
        for (uint64_t i = h.part_begin[q]; i < h.part_begin[q + 1]; ++i) out[q].push_back(hdp[i]);
    return out;
}

// computePartition<Sampler>(ptr, 2, dist) (misc.hpp:531-587 / 650-708) for
// every PE: interval_sizes[q][r] strings of PE q go to PE r.
inline std::vector<std::vector<size_t>> computePartition(Context& ctx,
                                                         const std::vector<std::vector<unsigned char>>& sorted_raw_per_pe,
                                                         const std::vector<std::vector<size_t>>& dp_per_pe,
                                                         Sampler s = Sampler::NumStrings) {
    HostArena h(sorted_raw_per_pe);
    DeviceArena d(h);
    std::vector<uint32_t> ord(h.n()), dp;
    for (size_t i = 0; i < h.n(); ++i) ord[i] = static_cast<uint32_t>(i);
    for (auto& v : dp_per_pe)
        for (size_t x : v) dp.push_back(static_cast<uint32_t>(x));
    if (dp.size() != h.n()) throw Error(DSSS_EINVAL, "one DP value per string expected");
    DeviceVec<uint32_t> dord(ord), ddp(dp);
    std::vector<uint64_t> iv((size_t)h.p() * h.p());
    dsss_opts o{static_cast<uint32_t>(s), 2, 0, 0};
    dsss_arena a = d.view();
    check(dsss_partition(ctx.get(), &a, h.p(), h.part_begin.data(), dord.p, ddp.p, &o, iv.data(), nullptr));
    std::vector<std::vector<size_t>> out(h.p());
    for (uint32_t q = 0; q < h.p(); ++q) out[q].assign(iv.begin() + (size_t)q * h.p(), iv.begin() + (size_t)(q + 1) * h.p());
    return out;
}

// XXHasher::hash(str, length, UINT64_MAX) (bloomfilter.hpp:1094-1102) for a
// batch of strings of one PE: hash of the first min(depth, length) bytes.
inline std::vector<uint64_t> xxhasher_hash(const std::vector<unsigned char>& raw, uint32_t depth) {
    HostArena h({raw});
    DeviceArena d(h);
    std::vector<uint32_t> ids(h.n());
    for (size_t i = 0; i < h.n(); ++i) ids[i] = static_cast<uint32_t>(i);
    DeviceVec<uint32_t> dids(ids);
    DeviceVec<uint64_t> out(h.n());
    dsss_arena a = d.view();
    check(dsss_prefix_hash(&a, dids.p, h.n(), depth, out.p, nullptr));
    check_cuda(cudaDeviceSynchronize());
    return out.host();
}

}  // namespace dsss_gpu
