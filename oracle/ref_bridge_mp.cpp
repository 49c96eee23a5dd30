// Test infrastructure: the reference's own distributed sorters, compiled from
// its sources where they lie and run as real ranks (processes) over the
// process-based MPI stand-in (oracle/shim_mpi), so that the oracle's
// restatements are pinned against the reference at p > 1.  Nothing in the
// product links this.
//
//   ref_mp pd  <input> <out>   DistributedPrefixDoublingSort::sort with the
//                               executable's default policies
//                               (src/executables/prefix_doubling.cpp:69-77,
//                               src/sorter/distributed/prefix_doubling.hpp:200-295)
//   ref_mp pdi <input> <out>   the same with SampleIndexedSplittersNumStringsPolicy
//   ref_mp ms  <input> <out>   DistributedMergeSort::sort with
//                               AllToAllStringImpl<..., EmptyLcpByteEncoderMemCpy>
//                               (src/sorter/distributed/lcp_aware_number_string_splitting.hpp:184-290)
//                               and extendPrefix, as executables/distributed_sorter.cpp:121-130 run them
//   ref_mp hq  <input> <out>   RQuick::sort as executables/HQuicksort.cpp:340-357 calls it
//
// Input (little-endian): u64 n, u64 p, u64 part_begin[p + 1], u64 char_bytes,
// then the n strings NUL-terminated back to back in index order.  Rank q
// sorts strings part_begin[q] .. part_begin[q + 1].  Output: <out>.<rank>,
// a sequence of u64 arrays, each prefixed by its element count:
//   pd/pdi: local order (local indices after radixsort_CI3), local LCPs,
//           distinguishing-prefix lengths (computeDistinguishingPrefixes, in
//           local sorted order), interval sizes (computePartition), and the
//           permutation returned by sort() as (stringIndex, PEIndex) pairs;
//   ms:     the merged strings' bytes (one u64 per byte) and their LCPs;
//   hq:     the PE's sorted strings' bytes (one u64 per byte, NUL-terminated).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mpi/environment.hpp"
#include "sorter/distributed/prefix_doubling.hpp"
#include "sorter/distributed/lcp_aware_number_string_splitting.hpp"
#include "sorter/RQuick/RQuick.hpp"

namespace {

using StringSet = dss_schimek::UCharLengthStringSet;
using StringLcpPtr = tlx::sort_strings_detail::StringLcpPtr<StringSet, size_t>;

struct Input {
    uint64_t n = 0, p = 0;
    std::vector<uint64_t> pb;
    std::vector<unsigned char> raw;    // this rank's strings, NUL-terminated
    std::vector<uint64_t> starts;      // start of each local string in raw
};

bool read_input(const char* path, uint32_t rank, Input& in) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    auto rd = [&](void* p, size_t b) { return std::fread(p, 1, b, f) == b; };
    uint64_t cb = 0;
    if (!rd(&in.n, 8) || !rd(&in.p, 8)) return false;
    in.pb.resize(in.p + 1);
    if (!rd(in.pb.data(), 8 * (in.p + 1)) || !rd(&cb, 8)) return false;
    std::vector<unsigned char> all(cb);
    if (!rd(all.data(), cb)) return false;
    std::fclose(f);
    uint64_t pos = 0, idx = 0;
    for (; idx < in.pb[rank]; ++idx) pos += std::strlen(reinterpret_cast<char*>(&all[pos])) + 1;
    for (; idx < in.pb[rank + 1]; ++idx) {
        uint64_t l = std::strlen(reinterpret_cast<char*>(&all[pos])) + 1;
        in.starts.push_back(in.raw.size());
        in.raw.insert(in.raw.end(), all.begin() + pos, all.begin() + pos + l);
        pos += l;
    }
    return true;
}

struct Out {
    FILE* f;
    void arr(const std::vector<uint64_t>& v) {
        uint64_t c = v.size();
        std::fwrite(&c, 8, 1, f);
        if (c) std::fwrite(v.data(), 8, c, f);
    }
};

template <typename Container>
std::vector<uint64_t> local_indices(const Container& cont, const std::vector<uint64_t>& starts) {
    std::vector<uint64_t> order;
    const unsigned char* base = cont.raw_strings().data();
    for (size_t i = 0; i < cont.size(); ++i) {
        uint64_t off = static_cast<uint64_t>(cont.strings()[i].string - base);
        order.push_back(static_cast<uint64_t>(std::lower_bound(starts.begin(), starts.end(), off) - starts.begin()));
    }
    return order;
}

template <typename Sampler>
void run_pd(Input& in, Out& out) {
    using namespace dss_schimek;
    // the stages one by one on a copy, for their intermediate results
    {
        StringLcpContainer<StringSet> cont(std::vector<unsigned char>(in.raw));
        StringLcpPtr ptr = cont.make_string_lcp_ptr();
        tlx::sort_strings_detail::radixsort_CI3(ptr, 0, 0);
        std::vector<uint64_t> order = local_indices(cont, in.starts), lcp(cont.size());
        for (size_t i = 0; i < cont.size(); ++i) lcp[i] = i == 0 ? 0 : cont.lcps()[i];
        std::vector<size_t> dp = computeDistinguishingPrefixes<StringLcpPtr, AllToAllHashesNaive>(ptr);
        std::vector<uint64_t> iv = computePartition<Sampler, StringLcpPtr>(ptr, 2, dp);
        out.arr(order);
        out.arr(lcp);
        out.arr(std::vector<uint64_t>(dp.begin(), dp.end()));
        out.arr(iv);
    }
    StringLcpContainer<StringSet> cont(std::move(in.raw));
    StringLcpPtr ptr = cont.make_string_lcp_ptr();
    using AllToAll = mpi::AllToAllStringImplPrefixDoubling<false, StringLcpPtr,
                                                           mpi::AllToAllvCombined<mpi::AllToAllvSmall>>;
    DistributedPrefixDoublingSort<StringLcpPtr, Sampler, AllToAll, AllToAllHashesNaive> sorter;
    std::vector<StringIndexPEIndex> perm = sorter.sort(std::move(cont), ptr);
    std::vector<uint64_t> flat;
    for (const auto& e : perm) {
        flat.push_back(e.stringIndex);
        flat.push_back(e.PEIndex);
    }
    out.arr(flat);
}

void run_ms(Input& in, Out& out) {
    using namespace dss_schimek;
    StringLcpContainer<StringSet> cont(std::move(in.raw));
    StringLcpPtr ptr = cont.make_string_lcp_ptr();
    using AllToAll = mpi::AllToAllStringImpl<false, StringSet, mpi::AllToAllvCombined<mpi::AllToAllvSmall>,
                                             EmptyLcpByteEncoderMemCpy>;
    DistributedMergeSort<StringLcpPtr, SampleSplittersNumStringsPolicy<StringSet>, AllToAll, false> sorter;
    StringLcpContainer<StringSet> res = sorter.sort(ptr, std::move(cont));
    // distributed_sorter.cpp:127-130: the received strings carry no prefix
    // until extendPrefix restores it
    if (AllToAll::PrefixCompression && mpi::environment().size() > 1)
        res.extendPrefix(res.make_string_set(), res.savedLcps());
    std::vector<uint64_t> bytes, lcps;
    for (size_t i = 0; i < res.size(); ++i) {
        const unsigned char* s = res.strings()[i].string;
        for (; *s; ++s) bytes.push_back(*s);
        bytes.push_back(0);
        lcps.push_back(i == 0 ? 0 : res.lcps()[i]);
    }
    out.arr(bytes);
    out.arr(lcps);
}

void run_hq(Input& in, Out& out, uint32_t rank) {
    using namespace dss_schimek;
    std::mt19937_64 generator;
    generator.seed(3469931 + rank);
    using StringContainer = dss_schimek::StringContainer<StringSet>;
    RQuick::Data<StringContainer, StringContainer::isIndexed> data;
    data.rawStrings = std::move(in.raw);
    MPI_Comm comm = MPI_COMM_WORLD;
    auto sorted = RQuick::sort(generator, std::move(data), MPI_BYTE, 11111, comm, StringComparator(), true);
    std::vector<uint64_t> bytes;
    for (size_t i = 0; i < sorted.size(); ++i) {
        const unsigned char* s = sorted.strings()[i].string;
        for (; *s; ++s) bytes.push_back(*s);
        bytes.push_back(0);
    }
    out.arr(bytes);
}

}  // namespace

int main(int argc, char** argv) {
    dss_schimek::mpi::environment env;
    if (argc != 4) {
        std::fprintf(stderr, "usage: ref_mp pd|pdi|ms|hq <input> <out>\n");
        env.finalize();
        return 1;
    }
    const std::string mode = argv[1];
    Input in;
    if (!read_input(argv[2], env.rank(), in) || in.p != env.size()) {
        std::fprintf(stderr, "ref_mp: bad input or rank count\n");
        MPI_Abort(MPI_COMM_WORLD, 1);
    }
    std::string path = std::string(argv[3]) + "." + std::to_string(env.rank());
    Out out{std::fopen(path.c_str(), "wb")};
    if (mode == "pd") run_pd<dss_schimek::SampleSplittersNumStringsPolicy<StringSet>>(in, out);
    else if (mode == "pdi") run_pd<dss_schimek::SampleIndexedSplittersNumStringsPolicy<StringSet>>(in, out);
    else if (mode == "ms") run_ms(in, out);
    else if (mode == "hq") run_hq(in, out, env.rank());
    std::fclose(out.f);
    env.barrier();
    env.finalize();
    return 0;
}
