// ORACLE — test infrastructure only.
//
// A single-process CPU restatement of the reference's prefix-doubling sample
// sort (DistributedPrefixDoublingSort, src/sorter/distributed/prefix_doubling.hpp:200-295)
// with p simulated PEs.  It is the checker for the CUDA path: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs
// may load it, and never as the thing measured for the product.
//
// Pinning: tests/test_oracle_pins.py checks every stage against code of the
// reference itself compiled in oracle/_ref (xxhash.hpp, tlx radixsort_CI3,
// BloomFilter/computeDistinguishingPrefixes at one PE, LcpStringLoserTree_)
// and against the reference's PD-exchange known-answer test
// (src/tests/alltoallStrings_tests.cpp:129-163) via tests/golden/.
// oracle_hq_sort (RQuick, the hQuicksort competitor) is unpinned against the
// reference's binary (RQuick needs MPI, not available here); its random bits
// come from std::mt19937_64 as the reference's do, and the tests check it
// against a second, pure-Python restatement with its own MT19937-64 (pinned
// to the C++ standard's known answer) and against the reference
// executable's own check (the PEs' outputs in rank order are the sorted input).
//
// Strings are (offset, length) views into one byte arena; bytes at or past a
// string's length read as 0, which is exactly the NUL terminator the
// reference's StringSets rely on.  Strings must not contain byte 0.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

namespace {

struct Arena {
    const uint8_t* chars;
    const uint64_t* off;
    const uint32_t* len;
    uint64_t n;
    inline uint8_t at(uint64_t s, uint64_t i) const { return i < len[s] ? chars[off[s] + i] : 0; }
};

// ---------------------------------------------------------------- XXH64 ----
// XXH64 with seed 0 as the reference's streaming port computes it
// (src/hash/xxhash.hpp:327-350 round/mergeRound, :516-600 update, :602-660 digest).
// The published XXH64 algorithm, with the port's one deviation: the four-lane
// merge is taken only when total_len > 32 (xxhash.hpp:608), so a 32-byte input
// hashes as v3 + PRIME5 after one stripe.
constexpr uint64_t P1 = 11400714785074694791ULL, P2 = 14029467366897019727ULL,
                   P3 = 1609587929392839161ULL, P4 = 9650029242287828579ULL,
                   P5 = 2870177450012600261ULL;
inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t rd64(const uint8_t* p) { uint64_t v; std::memcpy(&v, p, 8); return v; }
inline uint32_t rd32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; }
inline uint64_t xround(uint64_t acc, uint64_t in) { acc += in * P2; acc = rotl(acc, 31); return acc * P1; }
inline uint64_t xmerge(uint64_t acc, uint64_t v) { v = xround(0, v); acc ^= v; return acc * P1 + P4; }

uint64_t xxh64(const uint8_t* p, uint64_t len) {
    const uint8_t* const end = p + len;
    uint64_t v1 = P1 + P2, v2 = P2, v3 = 0, v4 = 0 - P1;
    if (len >= 32) {
        const uint8_t* const limit = end - 32;
        do {
            v1 = xround(v1, rd64(p)); v2 = xround(v2, rd64(p + 8));
            v3 = xround(v3, rd64(p + 16)); v4 = xround(v4, rd64(p + 24));
            p += 32;
        } while (p <= limit);
    }
    uint64_t h;
    if (len > 32) {
        h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
        h = xmerge(h, v1); h = xmerge(h, v2); h = xmerge(h, v3); h = xmerge(h, v4);
    } else {
        h = v3 + P5;
    }
    h += len;
    while (p + 8 <= end) { h ^= xround(0, rd64(p)); h = rotl(h, 27) * P1 + P4; p += 8; }
    if (p + 4 <= end) { h ^= (uint64_t)rd32(p) * P1; h = rotl(h, 23) * P2 + P3; p += 4; }
    while (p < end) { h ^= (uint64_t)(*p) * P5; h = rotl(h, 11) * P1; ++p; }
    h ^= h >> 33; h *= P2; h ^= h >> 29; h *= P3; h ^= h >> 32;
    return h;
}

// XXHasher::hash (bloomfilter.hpp:1095-1102): digest % bloomFilterSize with
// bloomFilterSize = UINT64_MAX (bloomfilter.hpp:1135).
inline uint64_t filter_hash(const Arena& a, uint64_t s, uint64_t depth) {
    return xxh64(a.chars + a.off[s], depth) % UINT64_MAX;
}

// ------------------------------------------------------ string compare ----
// scmp (strings/stringtools.hpp:128-136) on arena strings: <0, 0, >0.
inline int scmp(const Arena& a, uint64_t s, const uint8_t* t, uint64_t tlen) {
    uint64_t i = 0;
    for (;; ++i) {
        uint8_t x = a.at(s, i), y = i < tlen ? t[i] : 0;
        if (x == 0 || x != y) return (int)x - (int)y;
    }
}
inline uint64_t calc_lcp(const Arena& a, uint64_t s, uint64_t t) {
    uint64_t m = std::min(a.len[s], a.len[t]);
    const uint8_t* x = a.chars + a.off[s];
    const uint8_t* y = a.chars + a.off[t];
    uint64_t i = 0;
    while (i < m && x[i] == y[i]) ++i;
    return i;
}
inline bool str_less(const Arena& a, uint64_t s, uint64_t t) {
    uint64_t m = std::min(a.len[s], a.len[t]);
    int c = std::memcmp(a.chars + a.off[s], a.chars + a.off[t], m);
    if (c != 0) return c < 0;
    return a.len[s] < a.len[t];
}

// ------------------------------------------------------------ local sort ----
// radixsort_CI3 (tlx/sort/strings/radix_sort.hpp:861-884) result: the PE's
// strings in lexicographic order with lcp[i] = lcp(s_{i-1}, s_i), lcp[0] = 0.
// Byte-identical strings have no observable order in the reference; here they
// are kept in input order.
void local_sort(const Arena& a, uint32_t p, const uint64_t* pb, uint64_t* order, uint64_t* lcp) {
    for (uint32_t q = 0; q < p; ++q) {
        uint64_t b = pb[q], e = pb[q + 1];
        for (uint64_t i = b; i < e; ++i) order[i] = i;
        std::stable_sort(order + b, order + e, [&](uint64_t x, uint64_t y) { return str_less(a, x, y); });
        for (uint64_t i = b; i < e; ++i) lcp[i] = i == b ? 0 : calc_lcp(a, order[i - 1], order[i]);
    }
}

// ------------------------------------------------------------- DP rounds ----
struct HashStringIndex {  // bloomfilter.hpp:94-121
    uint64_t hashValue;
    uint64_t stringIndex;
    bool isLocalDuplicate = false;
    bool isLocalDuplicateButSendAnyway = false;
    bool isLcpLocalRoot = false;
};

struct PeView {  // one PE's locally sorted strings
    const Arena* a;
    const uint64_t* order;  // string ids in local order
    const uint64_t* lcp;
    uint64_t n;
    uint64_t len(uint64_t i) const { return a->len[order[i]]; }
};

struct Generated {
    std::vector<HashStringIndex> records;
    std::vector<uint64_t> localDups;
    std::vector<uint64_t> eos;
};

// generateHashStringIndices: round 0 (bloomfilter.hpp:1273-1331) when
// candidates == nullptr, later rounds (bloomfilter.hpp:1162-1227) otherwise.
Generated generate(const PeView& v, const std::vector<uint64_t>* candidates, uint64_t depth) {
    Generated g;
    uint64_t m = candidates ? candidates->size() : v.n;
    if (m == 0) return g;
    auto cand = [&](uint64_t j) { return candidates ? (*candidates)[j] : j; };
    for (uint64_t j = 0; j < m; ++j) {
        uint64_t c = cand(j);
        uint64_t L = v.len(c);
        if (depth > L) {
            g.eos.push_back(c);
        } else if (j > 0 && (candidates ? cand(j - 1) + 1 == c : true) && v.lcp[c] >= depth) {
            g.localDups.push_back(c);
            // records is never empty here: c-1 shares >= depth bytes with c, so it
            // was hashed or is itself an LCP duplicate of a hashed string.
            if (!g.records.empty() && g.records.back().stringIndex + 1 == c)
                g.records.back().isLcpLocalRoot = true;
        } else {
            g.records.push_back({filter_hash(*v.a, v.order[c], depth), c});
        }
    }
    return g;
}

// getIndicesOfLocalDuplicates (bloomfilter.hpp:1333-1378), including its
// final-element re-check (:1370-1376).
std::vector<uint64_t> local_hash_dups(std::vector<HashStringIndex>& r) {
    std::vector<uint64_t> out;
    if (r.empty()) return out;
    for (uint64_t i = 0; i < r.size() - 1;) {
        HashStringIndex& piv = r[i];
        uint64_t j = i + 1;
        HashStringIndex& cur = r[j];
        if (cur.hashValue == piv.hashValue) {
            piv.isLocalDuplicate = true;
            piv.isLocalDuplicateButSendAnyway = true;
            cur.isLocalDuplicate = true;
            out.push_back(piv.stringIndex);
            out.push_back(cur.stringIndex);
            ++j;
            while (j < r.size() && r[j].hashValue == piv.hashValue) {
                r[j].isLocalDuplicate = true;
                out.push_back(r[j].stringIndex);
                ++j;
            }
        } else if (piv.isLcpLocalRoot) {
            piv.isLocalDuplicate = true;
            piv.isLocalDuplicateButSendAnyway = true;
            out.push_back(piv.stringIndex);
        }
        i = j;
    }
    if (r.back().isLcpLocalRoot) {
        r.back().isLocalDuplicate = true;
        r.back().isLocalDuplicateButSendAnyway = true;
        out.push_back(r.back().stringIndex);
    }
    return out;
}

// One round of BloomFilter::filter over all PEs (bloomfilter.hpp:1415-1556):
// hashes are range-partitioned over p filter PEs (computeIntervalSizes :529-546),
// each filter PE merges its received sorted runs and reports every member of an
// equal-hash run back to its owner (FindDuplicates :662-765), and each owner
// merges remote, local-hash and LCP duplicates into its next candidate list
// (getSortedIndicesOfDuplicates :767-817).  setDepth (:1380-1411) writes results.
void filter_round(const std::vector<PeView>& pes, uint64_t depth,
                  std::vector<std::vector<uint64_t>>& candidates, bool first,
                  std::vector<std::vector<uint64_t>>& results) {
    const uint32_t p = (uint32_t)pes.size();
    std::vector<Generated> gen(p);
    std::vector<std::vector<uint64_t>> localHash(p);
    std::vector<std::vector<HashStringIndex>> reduced(p);
    for (uint32_t q = 0; q < p; ++q) {
        gen[q] = generate(pes[q], first ? nullptr : &candidates[q], depth);
        auto& r = gen[q].records;
        std::stable_sort(r.begin(), r.end(),
                         [](const HashStringIndex& x, const HashStringIndex& y) { return x.hashValue < y.hashValue; });
        localHash[q] = local_hash_dups(r);
        for (auto& h : r)
            if (!h.isLocalDuplicate || h.isLocalDuplicateButSendAnyway) reduced[q].push_back(h);
    }
    // computeIntervalSizes: slice k holds hashes <= (k+1)*(UINT64_MAX/p) - 1.
    std::vector<std::vector<uint64_t>> sliceBegin(p, std::vector<uint64_t>(p + 1));
    for (uint32_t q = 0; q < p; ++q) {
        auto& r = reduced[q];
        uint64_t pos = 0;
        sliceBegin[q][0] = 0;
        for (uint32_t k = 0; k + 1 < p; ++k) {
            uint64_t lim = (uint64_t)(k + 1) * (UINT64_MAX / p) - 1;
            while (pos < r.size() && r[pos].hashValue <= lim) ++pos;
            sliceBegin[q][k + 1] = pos;
        }
        sliceBegin[q][p] = r.size();
    }
    // filter PE f: duplicates among the hashes it received (positions are
    // indices into the owner's reduced list).
    std::vector<std::vector<uint64_t>> remote(p);
    for (uint32_t f = 0; f < p; ++f) {
        struct HP { uint64_t h; uint32_t pe; uint64_t pos; };
        std::vector<HP> merged;
        for (uint32_t q = 0; q < p; ++q)
            for (uint64_t i = sliceBegin[q][f]; i < sliceBegin[q][f + 1]; ++i)
                merged.push_back({reduced[q][i].hashValue, q, i});
        std::stable_sort(merged.begin(), merged.end(), [](const HP& x, const HP& y) { return x.h < y.h; });
        for (uint64_t i = 0; i < merged.size();) {
            uint64_t j = i + 1;
            while (j < merged.size() && merged[j].h == merged[i].h) ++j;
            if (j - i >= 2)
                for (uint64_t k = i; k < j; ++k) remote[merged[k].pe].push_back(merged[k].pos);
            i = j;
        }
    }
    for (uint32_t q = 0; q < p; ++q) {
        std::vector<uint64_t> rem;
        for (uint64_t pos : remote[q])
            if (!reduced[q][pos].isLocalDuplicateButSendAnyway) rem.push_back(reduced[q][pos].stringIndex);
        std::sort(rem.begin(), rem.end());
        auto& lh = localHash[q];
        std::sort(lh.begin(), lh.end());
        std::vector<uint64_t> next;
        next.reserve(lh.size() + gen[q].localDups.size() + rem.size());
        next.insert(next.end(), lh.begin(), lh.end());
        next.insert(next.end(), gen[q].localDups.begin(), gen[q].localDups.end());
        next.insert(next.end(), rem.begin(), rem.end());
        std::sort(next.begin(), next.end());
        // setDepth
        if (first) {
            std::fill(results[q].begin(), results[q].end(), depth);
        } else {
            for (uint64_t c : candidates[q]) results[q][c] = depth;
        }
        for (uint64_t c : gen[q].eos) results[q][c] = pes[q].len(c);
        candidates[q] = std::move(next);
    }
}

// computeDistinguishingPrefixes (prefix_doubling.hpp:156-198): depths
// 8, 8+16, 8+32, 8+64, ... until no PE has candidates left.
void dp_rounds(const Arena& a, uint32_t p, const uint64_t* pb, const uint64_t* order,
               const uint64_t* lcp, uint64_t* dp, uint64_t* round_counts, uint32_t max_rounds,
               uint32_t* rounds_out) {
    std::vector<PeView> pes(p);
    std::vector<std::vector<uint64_t>> results(p), cand(p);
    for (uint32_t q = 0; q < p; ++q) {
        pes[q] = {&a, order + pb[q], lcp + pb[q], pb[q + 1] - pb[q]};
        results[q].assign(pes[q].n, 0);
    }
    const uint64_t start = 8;
    uint32_t r = 0;
    filter_round(pes, start, cand, true, results);
    for (uint64_t i = start * 2;; i *= 2) {
        uint64_t total = 0;
        for (auto& c : cand) total += c.size();
        if (round_counts && r < max_rounds) round_counts[r] = total;
        ++r;
        if (total == 0) break;
        filter_round(pes, start + i, cand, false, results);
    }
    if (rounds_out) *rounds_out = r;
    for (uint32_t q = 0; q < p; ++q)
        for (uint64_t i = 0; i < pes[q].n; ++i) dp[pb[q] + i] = results[q][i];
}

// ------------------------------------------------------------- partition ----
// computePartition for the distinguishing-prefix path: non-indexed
// (misc.hpp:531-587 with SampleSplittersNumStringsPolicy, samplingStrategies.hpp:57-89)
// or indexed (misc.hpp:650-708 with SampleIndexedSplittersNumStringsPolicy,
// samplingStrategies.hpp:148-184).  The distributed sample sort (RQuick) is
// replaced by a sequential sort with the same comparator; getSplitters
// (misc.hpp:89-135/137-189) picks every (total/(nr+1))-th sorted sample.
struct Sample { std::vector<uint8_t> s; uint64_t index; };

void partition(const Arena& a, uint32_t p, const uint64_t* pb, const uint64_t* order,
               const uint64_t* dp, uint32_t sampling_factor, bool indexed, uint64_t* intervals) {
    std::vector<Sample> samples;
    for (uint32_t q = 0; q < p; ++q) {
        uint64_t nq = pb[q + 1] - pb[q];
        uint64_t nr = std::min<uint64_t>((uint64_t)sampling_factor * (p - 1), nq);  // getNumberSplitter
        double dist = (double)nq / (double)(nr + 1);
        for (uint64_t i = 1; i <= nr; ++i) {
            uint64_t idx = (uint64_t)(i * dist);
            uint64_t s = order[pb[q] + idx];
            uint64_t used = std::min<uint64_t>(a.len[s], dp[pb[q] + idx]);
            Sample sm;
            sm.s.assign(a.chars + a.off[s], a.chars + a.off[s] + used);
            sm.index = pb[q] + idx;  // localOffset + splitterIndex
            samples.push_back(std::move(sm));
        }
    }
    auto cmp = [&](const Sample& x, const Sample& y) {
        uint64_t m = std::min(x.s.size(), y.s.size());
        int c = m ? std::memcmp(x.s.data(), y.s.data(), m) : 0;
        if (c != 0) return c < 0;
        if (x.s.size() != y.s.size()) return x.s.size() < y.s.size();
        return indexed ? x.index < y.index : false;
    };
    std::stable_sort(samples.begin(), samples.end(), cmp);
    uint64_t total = samples.size();
    uint64_t nspl = std::min<uint64_t>(p - 1, total);
    uint64_t sdist = total / (nspl + 1);
    std::vector<const Sample*> spl;
    for (uint64_t i = 1; i <= nspl; ++i) spl.push_back(&samples[i * sdist]);
    for (uint32_t q = 0; q < p; ++q) {
        uint64_t nq = pb[q + 1] - pb[q];
        const uint64_t* ord = order + pb[q];
        std::vector<uint64_t> pos;
        for (const Sample* sp : spl) {
            // binarySearch (misc.hpp:310-333) / binarySearchIndexed (:347-374)
            uint64_t left = 0, right = nq, found = UINT64_MAX;
            while (left != right) {
                uint64_t d = (right - left) / 2;
                int res;
                if (!indexed) {
                    res = scmp(a, ord[left + d], sp->s.data(), sp->s.size());
                } else {
                    // indexStringCompare (misc.hpp:335-345)
                    uint64_t s = ord[left + d];
                    uint64_t i = 0;
                    uint8_t x, y;
                    for (;; ++i) {
                        x = a.at(s, i);
                        y = i < sp->s.size() ? sp->s[i] : 0;
                        if (!(x == y && x != 0)) break;
                    }
                    if (x != y) res = (int)x - (int)y;
                    else res = (int)(int64_t)((left + d + pb[q]) - sp->index);
                }
                if (res < 0) left = left + d + 1;
                else if (res == 0) { found = left + d; break; }
                else right = left + d;
            }
            pos.push_back(found != UINT64_MAX ? found : left);
        }
        pos.push_back(nq);
        for (uint64_t k = pos.size() - 1; k > 0; --k) pos[k] -= pos[k - 1];
        // fewer than p - 1 splitters (a sample smaller than p - 1): the last
        // bucket that has a splitter bound takes the rest, later ones none
        // (the reference's interval vector would be shorter than p there)
        for (uint32_t r = 0; r < p; ++r) intervals[(uint64_t)q * p + r] = r < pos.size() ? pos[r] : 0;
    }
}

// -------------------------------------------------------------- exchange ----
// AllToAllStringImplPrefixDoubling::alltoallv (mpi/alltoall.hpp:910-1008) with
// EmptyPrefixDoublingLcpByteEncoderMemCpy (mpi/byte_encoder.hpp:139-171):
// LCP := 0 at each non-empty interval start (setLcpAtStartOfInterval :396-404),
// each string sends bytes [lcp, dp) and a NUL.  PE r receives, in source order,
// the r-th interval of every PE; tags are (sender bucket offset + i, sender)
// (stringcontainer.hpp:127-158).
struct Recv {
    std::vector<uint8_t> chars;
    std::vector<uint64_t> lcp, index, pe, start;  // start: offset of each string in chars
    std::vector<uint64_t> counts, offsets;       // per source PE
};

std::vector<Recv> exchange(const Arena& a, uint32_t p, const uint64_t* pb, const uint64_t* order,
                           const uint64_t* lcp_in, const uint64_t* dp, const uint64_t* intervals) {
    std::vector<Recv> recv(p);
    for (auto& r : recv) { r.counts.assign(p, 0); r.offsets.assign(p, 0); }
    for (uint32_t q = 0; q < p; ++q) {
        uint64_t nq = pb[q + 1] - pb[q];
        std::vector<uint64_t> lcp(lcp_in + pb[q], lcp_in + pb[q] + nq);
        uint64_t it = 0;
        for (uint32_t r = 0; r < p; ++r) {
            uint64_t cnt = intervals[(uint64_t)q * p + r];
            if (cnt) lcp[it] = 0;
            it += cnt;
        }
        uint64_t off = 0;
        for (uint32_t r = 0; r < p; ++r) {
            uint64_t cnt = intervals[(uint64_t)q * p + r];
            Recv& R = recv[r];
            R.counts[q] = cnt;
            R.offsets[q] = off;
            for (uint64_t i = 0; i < cnt; ++i) {
                uint64_t li = off + i;
                uint64_t s = order[pb[q] + li];
                uint64_t l = lcp[li], d = dp[pb[q] + li];
                R.start.push_back(R.chars.size());
                for (uint64_t k = l; k < d; ++k) R.chars.push_back(a.chars[a.off[s] + k]);
                R.chars.push_back(0);
                R.lcp.push_back(l);
                R.index.push_back(off + i);
                R.pe.push_back(q);
            }
            off += cnt;
        }
    }
    return recv;
}

// ----------------------------------------------------------------- merge ----
// LcpStringLoserTree_<K> over one PE's receive container
// (merge/bingmann-lcp_losertree.hpp:203-480) driven as merge<K>
// (sorter/distributed/merging.hpp:23-63): K = pow2roundup(p) streams, empty
// padding streams, tree init with full-string games (updateNode :280-333,
// initTree :335-359), output loop with prefix-compressed games
// (updateNodeCompressedPrefix :225-278, writeElementsToStream :375-428).
struct LoserTree {
    struct Node { uint64_t idx, lcp; };
    struct Stream { uint64_t cur, end; };
    const Recv& R;
    uint64_t K;
    std::vector<Stream> streams;
    std::vector<Node> nodes;
    std::vector<uint64_t> lcpArr;  // the container's LCP array (range starts zeroed)

    LoserTree(const Recv& r, uint64_t k, const std::vector<std::pair<uint64_t, uint64_t>>& ranges)
        : R(r), K(k), streams(k + 1), nodes(k + 1), lcpArr(r.lcp) {
        for (uint64_t i = 1; i <= K; ++i) streams[i] = {ranges[i - 1].first, ranges[i - 1].first + ranges[i - 1].second};
        for (uint64_t k2 = 1; k2 <= K; ++k2) {
            Node c{k2, 0};
            uint64_t ni = K + k2;
            while (ni % 2 == 0 && ni > 2) { ni >>= 1; game(c, nodes[ni], false); }
            ni = (ni + 1) / 2;
            nodes[ni] = c;
        }
    }
    bool empty(uint64_t s) const { return streams[s].cur >= streams[s].end; }
    const uint8_t* chars(uint64_t s) const { return R.chars.data() + R.start[streams[s].cur]; }
    uint64_t firstLcp(uint64_t s) const { return lcpArr[streams[s].cur]; }
    void game(Node& contender, Node& defender, bool compressed) {
        if (empty(defender.idx)) return;
        if (empty(contender.idx)) { std::swap(defender, contender); return; }
        if (defender.lcp > contender.lcp) {
            std::swap(defender, contender);
        } else if (defender.lcp == contender.lcp) {
            uint64_t lcp = defender.lcp;
            const uint8_t* s1 = chars(defender.idx) + (compressed ? lcp - firstLcp(defender.idx) : lcp);
            const uint8_t* s2 = chars(contender.idx) + (compressed ? lcp - firstLcp(contender.idx) : lcp);
            while (*s1 != 0 && *s1 == *s2) ++s1, ++s2, ++lcp;
            if (*s1 < *s2) std::swap(defender, contender);
            defender.lcp = lcp;
        }
    }
    void run(uint64_t n, uint64_t* outPos, uint64_t* outLcp, uint64_t* outOld) {
        for (uint64_t o = 0; o < n; ++o) {
            uint64_t w = nodes[1].idx;
            outPos[o] = streams[w].cur;
            outLcp[o] = nodes[1].lcp;
            outOld[o] = firstLcp(w);
            ++streams[w].cur;
            Node& c = nodes[1];
            if (!empty(w)) c.lcp = firstLcp(w);
            uint64_t ni = w + K;
            while (ni > 2) { ni = (ni + 1) / 2; game(c, nodes[ni], true); }
        }
    }
};

void merge_one(const Recv& R, uint32_t p, uint64_t* idx, uint64_t* pe, uint64_t* lcp, uint64_t* old) {
    uint64_t n = R.lcp.size();
    if (n == 0) return;
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    uint64_t off = 0;
    for (uint32_t q = 0; q < p; ++q) {  // compute_ranges_and_set_lcp_at_start_of_range (misc.hpp:454-471)
        if (R.counts[q] == 0) { ranges.emplace_back(0, 0); continue; }
        ranges.emplace_back(off, R.counts[q]);
        off += R.counts[q];
    }
    uint64_t K = 1;
    while (K < p) K <<= 1;
    while (ranges.size() < K) ranges.emplace_back(0, 0);
    LoserTree t(R, K, ranges);
    std::vector<uint64_t> pos(n);
    t.run(n, pos.data(), lcp, old);
    for (uint64_t i = 0; i < n; ++i) { idx[i] = R.index[pos[i]]; pe[i] = R.pe[pos[i]]; }
}

}  // namespace

extern "C" {

uint64_t oracle_xxh64(const uint8_t* p, uint64_t len) { return xxh64(p, len); }

void oracle_local_sort(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n,
                       uint32_t p, const uint64_t* pb, uint64_t* order, uint64_t* lcp) {
    Arena a{chars, off, len, n};
    local_sort(a, p, pb, order, lcp);
}

// order/lcp: per-PE local sort output (as oracle_local_sort writes it).
void oracle_dp(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n,
               uint32_t p, const uint64_t* pb, const uint64_t* order, const uint64_t* lcp,
               uint64_t* dp, uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds) {
    Arena a{chars, off, len, n};
    dp_rounds(a, p, pb, order, lcp, dp, round_counts, max_rounds, rounds);
}

void oracle_partition(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n,
                      uint32_t p, const uint64_t* pb, const uint64_t* order, const uint64_t* dp,
                      uint32_t sampling_factor, int indexed, uint64_t* intervals) {
    Arena a{chars, off, len, n};
    partition(a, p, pb, order, dp, sampling_factor, indexed != 0, intervals);
}

// Exchange: writes the p receive containers back to back.  Sizes first:
// call with recv_chars == nullptr to get the total byte count in *char_total.
// Per string (n entries, destination-major): recv_lcp, recv_index, recv_pe;
// recv_char_begin[r] = first byte of PE r's container, [p] = total;
// recv_counts/recv_offsets [r*p + q]: strings PE r got from q, and q's bucket offset.
int oracle_exchange(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n,
                    uint32_t p, const uint64_t* pb, const uint64_t* order, const uint64_t* lcp,
                    const uint64_t* dp, const uint64_t* intervals, uint64_t* char_total,
                    uint8_t* recv_chars, uint64_t* recv_char_begin, uint64_t* recv_lcp,
                    uint64_t* recv_index, uint64_t* recv_pe, uint64_t* recv_counts,
                    uint64_t* recv_offsets) {
    Arena a{chars, off, len, n};
    std::vector<Recv> rv = exchange(a, p, pb, order, lcp, dp, intervals);
    uint64_t tot = 0;
    for (auto& r : rv) tot += r.chars.size();
    *char_total = tot;
    if (!recv_chars) return 0;
    uint64_t cb = 0, sb = 0;
    for (uint32_t r = 0; r < p; ++r) {
        recv_char_begin[r] = cb;
        std::memcpy(recv_chars + cb, rv[r].chars.data(), rv[r].chars.size());
        cb += rv[r].chars.size();
        for (uint64_t i = 0; i < rv[r].lcp.size(); ++i, ++sb) {
            recv_lcp[sb] = rv[r].lcp[i];
            recv_index[sb] = rv[r].index[i];
            recv_pe[sb] = rv[r].pe[i];
        }
        for (uint32_t q = 0; q < p; ++q) {
            recv_counts[(uint64_t)r * p + q] = rv[r].counts[q];
            recv_offsets[(uint64_t)r * p + q] = rv[r].offsets[q];
        }
    }
    recv_char_begin[p] = cb;
    return 0;
}

// Merge of one PE's receive container (chars of the prefix-compressed strings
// back to back, their sender-side LCPs, and per-source counts / bucket offsets).
int oracle_merge(const uint8_t* chars, uint64_t char_bytes, const uint64_t* lcps, uint64_t n, uint32_t p,
                 const uint64_t* counts, const uint64_t* offsets, uint64_t* idx, uint64_t* pe,
                 uint64_t* merged_lcp, uint64_t* old_lcp) {
    Recv R;
    R.chars.assign(chars, chars + char_bytes);
    R.counts.assign(counts, counts + p);
    R.offsets.assign(offsets, offsets + p);
    uint64_t pos = 0, k = 0;
    for (uint32_t q = 0; q < p; ++q)
        for (uint64_t i = 0; i < counts[q]; ++i, ++k) {
            if (k >= n || pos >= char_bytes) return -22;
            R.start.push_back(pos);
            R.lcp.push_back(lcps[k]);
            R.index.push_back(offsets[q] + i);
            R.pe.push_back(q);
            while (pos < char_bytes && chars[pos] != 0) ++pos;
            ++pos;
        }
    if (k != n) return -22;
    merge_one(R, p, idx, pe, merged_lcp, old_lcp);
    return 0;
}

// Full path.  Outputs (n entries each unless noted):
//   order, lcp: local sort per PE; dp: distinguishing prefixes in local order;
//   intervals [p*p]; perm_index/perm_pe/merged_lcp/old_lcp: merged output of
//   every PE back to back; recv_counts [p]: strings per destination PE.
// p == 1 stops after the local sort, as DistributedPrefixDoublingSort::sort
// does (prefix_doubling.hpp:236): recv_counts[0] = 0 and no permutation.
int oracle_pd_sort(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n,
                   uint32_t p, const uint64_t* pb, int indexed, uint64_t* order, uint64_t* lcp,
                   uint64_t* dp, uint64_t* intervals, uint64_t* perm_index, uint64_t* perm_pe,
                   uint64_t* merged_lcp, uint64_t* old_lcp, uint64_t* recv_counts) {
    Arena a{chars, off, len, n};
    local_sort(a, p, pb, order, lcp);
    if (p == 1) { recv_counts[0] = 0; return 0; }
    dp_rounds(a, p, pb, order, lcp, dp, nullptr, 0, nullptr);
    partition(a, p, pb, order, dp, 2, indexed != 0, intervals);
    std::vector<Recv> rv = exchange(a, p, pb, order, lcp, dp, intervals);
    uint64_t o = 0;
    for (uint32_t r = 0; r < p; ++r) {
        uint64_t m = rv[r].lcp.size();
        recv_counts[r] = m;
        merge_one(rv[r], p, perm_index + o, perm_pe + o, merged_lcp + o, old_lcp + o);
        o += m;
    }
    return 0;
}

// Merge-sort path: DistributedMergeSort::sort
// (sorter/distributed/lcp_aware_number_string_splitting.hpp:184-290) with the
// non-indexed sampler and AllToAllStringImpl<..., EmptyLcpByteEncoderMemCpy>
// (mpi/alltoall.hpp:724-804).  Local sort; avg = getAvgLcp (misc.hpp:68-87:
// the sum of every PE's local LCP array over the number of strings, integer
// division); computePartition(ptr, 100 * (avg + 5), 2) (misc.hpp:473-531)
// samples with SampleSplittersNumStringsPolicy's maxLength overload
// (samplingStrategies.hpp:25-55), each sample truncated to 2 * that = 200 *
// (avg + 5) bytes; the exchange sends whole strings LCP-compressed (bytes
// [lcp, length) and a NUL); choose_merge outputs every received string, whole,
// in order, with LCPs.  Outputs: order/lcp (local sort), intervals [p*p],
// source [n] (string id of every output string, receiving PEs back to back),
// out_lcp [n], recv_counts [p], *avg_lcp.  p == 1 returns the local sort
// (lcp_aware_number_string_splitting.hpp:230-232).
int oracle_ms_sort(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n, uint32_t p,
                   const uint64_t* pb, uint64_t* order, uint64_t* lcp, uint64_t* intervals, uint64_t* source,
                   uint64_t* out_lcp, uint64_t* recv_counts, uint64_t* avg_lcp) {
    Arena a{chars, off, len, n};
    local_sort(a, p, pb, order, lcp);
    uint64_t lsum = 0;
    for (uint64_t i = 0; i < n; ++i) lsum += lcp[i];
    const uint64_t avg = n ? lsum / n : 0;
    *avg_lcp = avg;
    if (p == 1) {
        for (uint64_t i = 0; i < n; ++i) {
            source[i] = order[i];
            out_lcp[i] = lcp[i];
        }
        intervals[0] = n;
        recv_counts[0] = n;
        return 0;
    }
    const uint64_t max_len = 2 * (100 * (avg + 5));
    std::vector<uint64_t> trunc(n ? n : 1, max_len), whole(n ? n : 1);
    for (uint64_t i = 0; i < n; ++i) whole[i] = len[order[i]];
    partition(a, p, pb, order, trunc.data(), 2, false, intervals);
    std::vector<Recv> rv = exchange(a, p, pb, order, lcp, whole.data(), intervals);
    uint64_t o = 0;
    for (uint32_t r = 0; r < p; ++r) {
        const uint64_t m = rv[r].lcp.size();
        recv_counts[r] = m;
        std::vector<uint64_t> idx(m ? m : 1), pe(m ? m : 1), ml(m ? m : 1), old(m ? m : 1);
        merge_one(rv[r], p, idx.data(), pe.data(), ml.data(), old.data());
        for (uint64_t k = 0; k < m; ++k, ++o) {
            source[o] = order[pb[pe[k]] + idx[k]];
            out_lcp[o] = ml[k];
        }
    }
    return 0;
}

// --------------------------------------------------------------- RQuick ----
// RQuick::sort as the hQuicksort executable runs it
// (src/executables/HQuicksort.cpp:307-358: robust, non-indexed strings, PE r's
// std::mt19937_64 seeded with 3469931 + r at :344-345) on p simulated PEs:
// sorter/RQuick/RQuick.hpp:834-1104 (sort) and :415-627 (sortRec).  The PEs'
// string lists hold string ids; strings compare as the executable's
// StringComparator (HQuicksort.cpp:27-42) does: bytes until the first
// difference or NUL.
int oracle_hq_sort(const uint8_t* chars, const uint64_t* off, const uint32_t* len, uint64_t n, uint32_t p,
                   const uint64_t* pb, uint64_t seed, uint64_t* source, uint64_t* counts) {
    (void)n;
    // a string, or the empty pivot getRawString(-1) returns (stringcontainer.hpp:582-585)
    struct Key { const uint8_t* c; uint32_t l; };
    auto key = [&](uint64_t id) { return Key{chars + off[id], len[id]}; };
    auto less = [](const Key& x, const Key& y) {
        const uint32_t m = std::min(x.l, y.l);
        const int c = m ? std::memcmp(x.c, y.c, m) : 0;
        return c ? c < 0 : x.l < y.l;
    };
    auto id_less = [&](uint64_t x, uint64_t y) { return less(key(x), key(y)); };
    std::vector<std::vector<uint64_t>> pe(p);
    for (uint32_t q = 0; q < p; ++q)
        for (uint64_t i = pb[q]; i < pb[q + 1]; ++i) pe[q].push_back(i);
    uint32_t pw = 1;
    while (pw * 2 <= p) pw *= 2;
    // PEs past the largest power of two hand their strings down (RQuick.hpp:878-959)
    for (uint32_t q = pw; q < p; ++q) {
        pe[q - pw].insert(pe[q - pw].end(), pe[q].begin(), pe[q].end());
        pe[q].clear();
    }
    for (uint32_t q = 0; q < pw; ++q) std::sort(pe[q].begin(), pe[q].end(), id_less);  // sortLocally
    // RandomBitStore (RandomBitStore.hpp:27-52): 64 bits per draw, lowest first
    struct Bits {
        std::mt19937_64 gen;
        uint64_t bits = 0;
        int pos = 64;
        uint64_t next() {
            if (pos == 64) { bits = gen(); pos = 0; }
            const uint64_t r = bits & 1;
            bits >>= 1;
            ++pos;
            return r;
        }
    };
    std::vector<Bits> bs(pw);
    for (uint32_t q = 0; q < pw; ++q) bs[q].gen.seed(seed + q);
    std::vector<uint64_t> beg(pw), sep(pw);
    for (uint32_t P = pw; P >= 2; P /= 2) {  // one level per halving of the subcube (:600-623)
        for (uint32_t b = 0; b < pw; b += P) {
            // selectSplitter: every PE's two middle-most strings (middleMostElements, RQuick.hpp:273-314)
            for (uint32_t q = b; q < b + P; ++q) {
                const uint64_t c = pe[q].size();
                beg[q] = c > 2 ? (c - 2) / 2 + (c % 2 == 1 ? bs[q].next() : 0) : 0;
            }
            // BinTreeMedianSelection::select (BinTreeMedianSelection.hpp:157-226):
            // selectMedians builds both of its containers from its own input
            // (:61-62; the second is the moved-from, empty vector), so the
            // medians received are dropped and the subcube's first PE picks
            // among its own (selectMedian :135-152: one of two by a bit)
            const uint64_t m = std::min<uint64_t>(pe[b].size(), 2);
            Key piv{chars, 0};
            if (m) piv = key(pe[b][beg[b] + (m == 2 ? bs[b].next() : 0)]);
            // locateSplitter, robust (RQuick.hpp:363-385)
            for (uint32_t q = b; q < b + P; ++q) {
                const std::vector<uint64_t>& v = pe[q];
                const uint64_t c = v.size();
                const uint64_t lo = std::lower_bound(v.begin(), v.end(), piv, [&](uint64_t x, const Key& k) {
                                        return less(key(x), k);
                                    }) - v.begin();
                const uint64_t hi = std::upper_bound(v.begin() + lo, v.end(), piv, [&](const Key& k, uint64_t x) {
                                        return less(k, key(x));
                                    }) - v.begin();
                const uint64_t opt = c / 2 + (c % 2 == 1 ? bs[q].next() : 0);
                sep[q] = lo < opt ? std::min(opt, hi) : lo;
            }
            // the left half keeps the small strings, the right half the large;
            // each merges what its partner sends after its own (RQuick.hpp:496-586)
            std::vector<std::vector<uint64_t>> next(P);
            for (uint32_t q = b; q < b + P; ++q) {
                const uint32_t r = b + (q - b + P / 2) % P;
                const bool left = q - b < P / 2;
                const std::vector<uint64_t>& v = pe[q];
                const std::vector<uint64_t>& w = pe[r];
                std::vector<uint64_t> own = left ? std::vector<uint64_t>(v.begin(), v.begin() + sep[q])
                                                 : std::vector<uint64_t>(v.begin() + sep[q], v.end());
                std::vector<uint64_t> got = left ? std::vector<uint64_t>(w.begin(), w.begin() + sep[r])
                                                 : std::vector<uint64_t>(w.begin() + sep[r], w.end());
                next[q - b].resize(own.size() + got.size());
                std::merge(own.begin(), own.end(), got.begin(), got.end(), next[q - b].begin(), id_less);
            }
            for (uint32_t q = b; q < b + P; ++q) pe[q] = std::move(next[q - b]);
        }
    }
    uint64_t o = 0;
    for (uint32_t q = 0; q < p; ++q) {
        counts[q] = pe[q].size();
        for (uint64_t id : pe[q]) source[o++] = id;
    }
    return 0;
}

}  // extern "C"

// --------------------------------------------------------------- Golomb ----
// The Golomb/delta coding of sorted 64-bit values that the reference's
// sequentialGolombEncoding policy applies to the hash exchange
// (AllToAllHashesGolomb, src/sorter/distributed/bloomfilter.hpp:164-313):
// per destination with c > 0 values the block is
//   [S, b, v_0, bit words...]   S = number of words after S,
// the bit words holding, for i = 1..c-1, the Golomb code of v_i - v_{i-1}
// most significant bit first (getDeltaEncoding, encoding/golomb_encoding.hpp:
// 61-80; DeltaStreamWriter, delta_stream.hpp:24-48; GolombBitStreamWriter::
// PutGolomb, golomb_bit_stream.hpp:59-115; BitStreamWriter::PutBits,
// bit_stream.hpp:52-83): q = delta / b ones, a zero, then r = delta mod b in
// truncated binary (k = ceil(log2 b) bits when r >= 2^k - b, stored as
// r + 2^k - b, else k - 1 bits); the last word's unused bits are ones (the
// writer's destructor, golomb_bit_stream.hpp:48-56).  A destination with no
// values gets no words.
static uint64_t golomb_param(uint64_t max_value, uint64_t count) {  // getB, golomb_encoding.hpp:50-59
    if (count == 0) return 1;
    const uint64_t avg = max_value / count;
    if (avg < 1) return 1;
    const uint64_t k = static_cast<uint64_t>(std::floor(std::log2(static_cast<double>(avg))));
    return 1ull << k;
}

static unsigned ceil_log2(uint64_t b) {  // tlx::integer_log2_ceil
    unsigned k = 0;
    while (k < 64 && (1ull << k) < b) ++k;
    return k;
}

namespace {
struct BitSink {  // most significant bit first into 64-bit words
    std::vector<uint64_t>& out;
    uint64_t cur = 0;
    unsigned used = 0;
    explicit BitSink(std::vector<uint64_t>& o) : out(o) {}
    void bit(unsigned v) {
        cur |= (uint64_t)(v & 1u) << (63 - used);
        if (++used == 64) {
            out.push_back(cur);
            cur = 0;
            used = 0;
        }
    }
    void bits(uint64_t v, unsigned k) {
        for (unsigned j = k; j-- > 0;) bit((unsigned)(v >> j) & 1u);
    }
    void ones(uint64_t q) {
        while (q && used) { bit(1); --q; }
        while (q >= 64) { out.push_back(~0ull); q -= 64; }
        while (q) { bit(1); --q; }
    }
    void finish() {  // the rest of a started word: ones
        if (used) {
            cur |= used ? (~0ull >> used) : 0;
            out.push_back(cur);
            cur = 0;
            used = 0;
        }
    }
};
}  // namespace

static void golomb_block(const uint64_t* v, uint64_t c, uint64_t b, std::vector<uint64_t>& out) {
    const size_t at = out.size();
    out.push_back(0);  // S, filled below
    out.push_back(b);
    out.push_back(v[0]);  // the first value is not coded
    const unsigned k = ceil_log2(b);
    const uint64_t little = (k >= 64 ? 0ull : (1ull << k)) - b;
    BitSink w(out);
    for (uint64_t i = 1; i < c; ++i) {
        const uint64_t d = v[i] - v[i - 1];
        const uint64_t q = d / b, r = d - q * b;
        w.ones(q);
        w.bit(0);
        if (r >= little) w.bits(r + little, k);
        else w.bits(r, k - 1);
    }
    w.finish();
    out[at] = out.size() - at - 1;
}

extern "C" {

uint64_t oracle_golomb_param(uint64_t max_value, uint64_t count) { return golomb_param(max_value, count); }

// b of the hash exchange to one of p PEs holding count hashes
// (bloomfilter.hpp:194-197: getB over the PE's slice of the 64-bit filter,
// bloomFilterSize = 2^64 - 1 at :1135, and 1 replaced by 20000000000).
uint64_t oracle_golomb_param_hashes(uint64_t count, uint32_t p) {
    const uint64_t b = golomb_param(~0ull / p, count);
    return b == 1 ? 20000000000ull : b;
}

// Blocks of nranges ranges (counts[r] sorted values each, back to back in
// values) with parameters b[r]; range_words[r] = the block's words (0 for an
// empty range).  Returns the total, -1 when it exceeds cap.
int64_t oracle_golomb_encode(const uint64_t* values, const uint64_t* counts, uint32_t nranges, const uint64_t* b,
                             uint64_t* out, uint64_t cap, uint64_t* range_words) {
    std::vector<uint64_t> w;
    uint64_t off = 0;
    for (uint32_t r = 0; r < nranges; ++r) {
        const size_t before = w.size();
        if (counts[r]) golomb_block(values + off, counts[r], b[r], w);
        range_words[r] = w.size() - before;
        off += counts[r];
    }
    if (w.size() > cap) return -1;
    std::copy(w.begin(), w.end(), out);
    return (int64_t)w.size();
}

// Decodes back-to-back blocks (nwords words) as the receiving side does
// (bloomfilter.hpp:230-242: per block S, b, then getDeltaDecoding until the
// bit reader finds no further zero); block_counts[k] = values of block k
// (at most max_blocks blocks).  Returns the values written, -1 on a
// malformed block or more than cap values.
int64_t oracle_golomb_decode(const uint64_t* words, uint64_t nwords, uint64_t* out, uint64_t cap,
                             uint64_t* block_counts, uint32_t max_blocks, uint32_t* nblocks) {
    uint64_t pos = 0, n = 0;
    uint32_t blk = 0;
    while (pos < nwords) {
        if (blk >= max_blocks) return -1;
        const uint64_t S = words[pos];
        if (S < 2 || S > nwords - pos - 1) return -1;
        const uint64_t end = pos + 1 + S, b = words[pos + 1];
        if (b == 0) return -1;
        const unsigned k = ceil_log2(b);
        const uint64_t little = (k >= 64 ? 0ull : (1ull << k)) - b;
        const uint64_t base = n;
        if (n >= cap) return -1;
        uint64_t v = words[pos + 2];
        out[n++] = v;
        const uint64_t bit0 = (pos + 3) * 64, bit1 = end * 64;
        auto get = [&](uint64_t t) -> unsigned { return (unsigned)(words[t >> 6] >> (63 - (t & 63))) & 1u; };
        uint64_t t = bit0;
        for (;;) {
            uint64_t q = 0;
            while (t < bit1 && get(t)) { ++q; ++t; }
            if (t >= bit1) break;  // only ones left: the padding
            ++t;  // the zero
            uint64_t r = 0;
            const unsigned lo = k ? k - 1 : 0;
            for (unsigned j = 0; j < lo; ++j) r = (r << 1) | (t < bit1 ? get(t++) : (t++, 0u));
            if (k && r >= little) r = ((r << 1) | (t < bit1 ? get(t++) : (t++, 0u))) - little;
            if (t > bit1) return -1;
            if (n >= cap) return -1;
            v += q * b + r;
            out[n++] = v;
        }
        block_counts[blk++] = n - base;
        pos = end;
    }
    *nblocks = blk;
    return (int64_t)n;
}

}  // extern "C"
