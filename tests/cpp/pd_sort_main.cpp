// Drives include/dsss_policies.hpp the way the reference's prefix_doubling
// executable drives DistributedPrefixDoublingSort: strings per PE in, local
// order / DP / intervals / permutation out, DistributedMergeSort and RQuick the way
// the merge-sort executable does (strings and LCPs per receiving PE).  Input (stdin): p, then for each
// PE a count and that many hex-encoded strings.  Output: one line per item.
#include <iostream>
#include <string>
#include <vector>

#include "dsss_policies.hpp"

static std::vector<unsigned char> unhex(const std::string& s) {
    std::vector<unsigned char> v;
    for (size_t i = 0; i + 1 < s.size(); i += 2) v.push_back((unsigned char)std::stoi(s.substr(i, 2), nullptr, 16));
    return v;
}

int main(int argc, char** argv) {
    int sampler = argc > 1 ? std::atoi(argv[1]) : 0;
    uint32_t p;
    std::cin >> p;
    std::vector<std::vector<unsigned char>> raw(p);
    for (uint32_t q = 0; q < p; ++q) {
        size_t m;
        std::cin >> m;
        for (size_t i = 0; i < m; ++i) {
            std::string h;
            std::cin >> h;
            if (h == "-") h.clear();
            auto s = unhex(h);
            raw[q].insert(raw[q].end(), s.begin(), s.end());
            raw[q].push_back(0);
        }
    }
    try {
        dsss_gpu::Context ctx(0);
        dsss_gpu::DistributedPrefixDoublingSort sorter(sampler == 2 ? dsss_gpu::Sampler::IndexedNumStrings
                                                                    : dsss_gpu::Sampler::NumStrings);
        auto r = sorter.sort(ctx, raw);
        for (uint32_t q = 0; q < p; ++q) {
            std::cout << "order " << q;
            for (auto x : r.local_order[q]) std::cout << ' ' << x;
            std::cout << "\ndp " << q;
            for (auto x : r.dp[q]) std::cout << ' ' << x;
            std::cout << "\nintervals " << q;
            for (auto x : r.interval_sizes[q]) std::cout << ' ' << x;
            std::cout << "\nperm " << q;
            for (auto x : r.permutation[q]) std::cout << ' ' << x.stringIndex << ':' << x.PEIndex;
            std::cout << "\nlcp " << q;
            for (auto x : r.merged_lcp[q]) std::cout << ' ' << x;
            std::cout << '\n';
        }
        // the merge-sort path: every receiving PE's strings (hex) and LCPs
        dsss_gpu::DistributedMergeSort ms;
        auto m = ms.sort(ctx, raw);
        std::cout << "msavg 0 " << m.avg_lcp << '\n';
        for (uint32_t q = 0; q < p; ++q) {
            std::cout << "msintervals " << q;
            for (auto x : m.interval_sizes[q]) std::cout << ' ' << x;
            std::cout << "\nmsstr " << q;
            std::string cur;
            for (unsigned char c : m.raw_strings[q]) {
                if (c == 0) {
                    std::cout << ' ' << (cur.empty() ? std::string("-") : cur);
                    cur.clear();
                } else {
                    static const char* hx = "0123456789abcdef";
                    cur += hx[c >> 4];
                    cur += hx[c & 15];
                }
            }
            std::cout << "\nmslcp " << q;
            for (auto x : m.lcps[q]) std::cout << ' ' << x;
            std::cout << '\n';
        }
        // hQuicksort: every PE's strings (hex)
        dsss_gpu::RQuick hq;
        auto hqs = hq.sort(ctx, raw);
        for (uint32_t q = 0; q < p; ++q) {
            std::cout << "hqstr " << q;
            std::string cur;
            for (unsigned char c : hqs[q]) {
                if (c == 0) {
                    std::cout << ' ' << (cur.empty() ? std::string("-") : cur);
                    cur.clear();
                } else {
                    static const char* hx = "0123456789abcdef";
                    cur += hx[c >> 4];
                    cur += hx[c & 15];
                }
            }
            std::cout << '\n';
        }
        // the stage adaptors on PE 0
        std::vector<std::vector<size_t>> order, lcp;
        dsss_gpu::radixsort_CI3(ctx, raw, order, lcp);
        std::cout << "ci3order";
        for (auto x : order[0]) std::cout << ' ' << x;
        std::cout << "\nci3lcp";
        for (auto x : lcp[0]) std::cout << ' ' << x;
        std::cout << '\n';
    } catch (const dsss_gpu::Error& e) {
        std::cerr << "error " << e.code << ": " << e.what() << '\n';
        return 2;
    }
    return 0;
}
