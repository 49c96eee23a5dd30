// Test infrastructure: C entry points over pieces of the reference itself,
// compiled from the reference's own headers where they lie (see oracle/Makefile),
// so the oracle restatement in oracle/oracle.cpp can be checked against the
// reference's code on the same inputs.  Nothing in the product links this.
//
// Pieces used (all header-only in the reference, none needs MPI):
//   src/hash/xxhash.hpp:508-706           xxh::hash_state_t<64> (XXH64, RedSpah port)
//   tlx/sort/strings/radix_sort.hpp:861   radixsort_CI3 (vendored tlx 2018-10-25)
//   src/strings/stringcontainer.hpp:163   StringLcpContainer + InitPolicy<IndexPEIndex> :127-158
//   src/merge/bingmann-lcp_losertree.hpp:203-480  LcpStringLoserTree_ (compressed-prefix merge)
//   src/sorter/distributed/merging.hpp:23-63  range padding of merge<K> (restated: the
//   header itself pulls in MPI)
//   src/encoding/golomb_encoding.hpp:50-110   getB, getDeltaEncoding / getDeltaDecoding over
//   thrill's Golomb bit streams (golomb_bit_stream.hpp, bit_stream.hpp, delta_stream.hpp);
//   the [S, b] block framing of AllToAllHashesGolomb (bloomfilter.hpp:199-209) is restated
//   here, since that struct's header pulls in MPI
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <numeric>
#include <vector>

#include "hash/xxhash.hpp"
#include "strings/stringcontainer.hpp"
#include "strings/stringset.hpp"
#include "merge/bingmann-lcp_losertree.hpp"
#include "encoding/golomb_encoding.hpp"
#include <tlx/sort/strings/radix_sort.hpp>

extern "C" {

uint64_t ref_xxh64(const uint8_t* data, uint64_t len) {
    xxh::hash_state_t<64> st;
    static const uint8_t empty = 0;
    st.update(len ? data : &empty, len);
    return st.digest();
}

// Local sort of n NUL-terminated strings laid out back to back in raw.
// order[i] = input index of the i-th smallest string, lcp[i] = LCP with i-1 (lcp[0] = 0).
int ref_radixsort_ci3(const uint8_t* raw, uint64_t raw_bytes, uint64_t n,
                      uint64_t* order, uint64_t* lcp) {
    using StringSet = dss_schimek::UCharLengthStringSet;
    std::vector<unsigned char> buf(raw, raw + raw_bytes);
    std::vector<uint64_t> starts;
    starts.reserve(n);
    for (uint64_t i = 0; i < raw_bytes;) {
        starts.push_back(i);
        while (buf[i] != 0) ++i;
        ++i;
    }
    if (starts.size() != n) return -22;
    dss_schimek::StringLcpContainer<StringSet> cont(std::move(buf));
    if (cont.size() != n) return -22;
    auto ptr = cont.make_string_lcp_ptr();
    tlx::sort_strings_detail::radixsort_CI3(ptr, 0, 0);
    const unsigned char* base = cont.raw_strings().data();
    auto* strs = cont.strings();
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t off = static_cast<uint64_t>(strs[i].string - base);
        auto it = std::lower_bound(starts.begin(), starts.end(), off);
        order[i] = static_cast<uint64_t>(it - starts.begin());
        lcp[i] = i == 0 ? 0 : cont.lcps()[i];
    }
    return 0;
}

} // extern "C"

template <size_t K>
static void run_losertree(dss_schimek::StringLcpContainer<dss_schimek::UCharIndexPEIndexStringSet>& cont,
                          std::vector<std::pair<size_t, size_t>>& ranges, uint64_t n,
                          uint64_t* out_index, uint64_t* out_pe, uint64_t* out_lcp,
                          uint64_t* out_oldlcp) {
    using StringSet = dss_schimek::UCharIndexPEIndexStringSet;
    std::vector<typename StringSet::String> sorted(n);
    std::vector<size_t> sorted_lcp(n);
    StringSet ss = cont.make_string_set();
    dss_schimek::StringLcpPtrMergeAdapter<StringSet> in(ss, cont.lcp_array());
    dss_schimek::LcpStringLoserTree_<K, StringSet> tree(in, ranges.data());
    StringSet outset(sorted.data(), sorted.data() + n);
    dss_schimek::StringLcpPtrMergeAdapter<StringSet> out(outset, sorted_lcp.data());
    std::vector<size_t> old;
    tree.writeElementsToStream(out, n, old);
    for (uint64_t i = 0; i < n; ++i) {
        out_index[i] = sorted[i].stringIndex;
        out_pe[i] = sorted[i].PEIndex;
        out_lcp[i] = sorted_lcp[i];
        out_oldlcp[i] = old[i];
    }
}

extern "C" {

// Merge of one PE's receive container (prefix-compressed strings, the layout
// AllToAllStringImplPrefixDoubling delivers): raw holds the strings of all
// sources back to back, lcps their sender-side LCPs, recv_counts/recv_offsets
// the per-source string counts and the senders' bucket offsets.
int ref_lcp_merge(const uint8_t* raw, uint64_t raw_bytes, const uint64_t* lcps, uint64_t n,
                  uint32_t p, const uint64_t* recv_counts, const uint64_t* recv_offsets,
                  uint64_t* out_index, uint64_t* out_pe, uint64_t* out_lcp,
                  uint64_t* out_oldlcp) {
    using StringSet = dss_schimek::UCharIndexPEIndexStringSet;
    if (n == 0) return 0;
    std::vector<unsigned char> buf(raw, raw + raw_bytes);
    std::vector<size_t> lc(lcps, lcps + n);
    std::vector<size_t> counts(recv_counts, recv_counts + p);
    std::vector<size_t> offs(recv_offsets, recv_offsets + p);
    dss_schimek::StringLcpContainer<StringSet> cont(std::move(buf), std::move(lc), counts, offs);
    if (cont.size() != n) return -22;
    // compute_ranges_and_set_lcp_at_start_of_range (misc.hpp:454-471)
    std::vector<std::pair<size_t, size_t>> ranges;
    for (size_t i = 0, offset = 0; i < p; ++i) {
        if (counts[i] == 0) { ranges.emplace_back(0, 0); continue; }
        cont.lcp_array()[offset] = 0;
        ranges.emplace_back(offset, counts[i]);
        offset += counts[i];
    }
    size_t K = 1;
    while (K < p) K <<= 1;  // pow2roundup (merging.hpp:10-21)
    for (size_t i = p; i < K; ++i) ranges.emplace_back(0u, 0u);
    switch (K) {
    case 1: run_losertree<1>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 2: run_losertree<2>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 4: run_losertree<4>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 8: run_losertree<8>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 16: run_losertree<16>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 32: run_losertree<32>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 64: run_losertree<64>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 128: run_losertree<128>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    case 256: run_losertree<256>(cont, ranges, n, out_index, out_pe, out_lcp, out_oldlcp); break;
    default: return -95;
    }
    return 0;
}

// getB (golomb_encoding.hpp:50-59).
uint64_t ref_golomb_param(uint64_t max_value, uint64_t count) { return getB(max_value, count); }

// One block as AllToAllHashesGolomb frames it: [S, b, getDeltaEncoding of
// the c values with parameter b].  Returns its words, -1 past cap.
int64_t ref_golomb_block(const uint64_t* values, uint64_t c, uint64_t b, uint64_t* out, uint64_t cap) {
    std::vector<size_t> enc;
    enc.push_back(0);
    enc.push_back(b);
    std::vector<size_t> v(values, values + c);
    getDeltaEncoding(v.begin(), v.end(), std::back_inserter(enc), b);
    enc[0] = enc.size() - 1;
    if (enc.size() > cap) return -1;
    std::copy(enc.begin(), enc.end(), out);
    return (int64_t)enc.size();
}

// One block's values: getDeltaDecoding over the words after S and b.
int64_t ref_golomb_unblock(const uint64_t* words, uint64_t nwords, uint64_t* out, uint64_t cap) {
    if (nwords < 3) return -1;
    std::vector<size_t> w(words, words + nwords);
    const size_t S = w[0], b = w[1];
    if (S + 1 != nwords) return -1;
    std::vector<size_t> dec;
    getDeltaDecoding(w.begin() + 2, w.end(), std::back_inserter(dec), b);
    if (dec.size() > cap) return -1;
    std::copy(dec.begin(), dec.end(), out);
    return (int64_t)dec.size();
}

} // extern "C"
