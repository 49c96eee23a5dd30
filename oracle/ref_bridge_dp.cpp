// Test infrastructure: the reference's own distinguishing-prefix computation,
// compiled from its headers where they lie with a ONE-rank MPI stand-in
// (oracle/shim_mpi1/mpi.h).  With one PE every exchange in BloomFilter::filter
// is a local copy, and the distinguishing-prefix lengths do not depend on how
// strings are split over PEs, so this pins the oracle's DP rounds for a whole
// string set.  Nothing in the product links this.
//
//   src/sorter/distributed/prefix_doubling.hpp:156-198  computeDistinguishingPrefixes
//   src/sorter/distributed/bloomfilter.hpp:1114-1557     BloomFilter (XXHasher, exact 64-bit dedup)
//   tlx/sort/strings/radix_sort.hpp:861                  radixsort_CI3 (the local sort before it)
#include <cstdint>
#include <algorithm>
#include <vector>

#include "sorter/distributed/prefix_doubling.hpp"

extern "C" int ref_dp_single_pe(const uint8_t* raw, uint64_t raw_bytes, uint64_t n,
                                uint64_t* order, uint64_t* lcp, uint64_t* dp) {
    using StringSet = dss_schimek::UCharLengthStringSet;
    using StringLcpPtr = tlx::sort_strings_detail::StringLcpPtr<StringSet, size_t>;
    std::vector<unsigned char> buf(raw, raw + raw_bytes);
    std::vector<uint64_t> starts;
    for (uint64_t i = 0; i < raw_bytes;) {
        starts.push_back(i);
        while (buf[i] != 0) ++i;
        ++i;
    }
    if (starts.size() != n) return -22;
    dss_schimek::StringLcpContainer<StringSet> cont(std::move(buf));
    StringLcpPtr ptr = cont.make_string_lcp_ptr();
    tlx::sort_strings_detail::radixsort_CI3(ptr, 0, 0);
    std::vector<size_t> res =
        dss_schimek::computeDistinguishingPrefixes<StringLcpPtr, dss_schimek::AllToAllHashesNaive>(ptr);
    const unsigned char* base = cont.raw_strings().data();
    auto* strs = cont.strings();
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t off = static_cast<uint64_t>(strs[i].string - base);
        order[i] = static_cast<uint64_t>(std::lower_bound(starts.begin(), starts.end(), off) - starts.begin());
        lcp[i] = i == 0 ? 0 : cont.lcps()[i];
        dp[i] = res[i];
    }
    return 0;
}
