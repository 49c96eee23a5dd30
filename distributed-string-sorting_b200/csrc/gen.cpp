// Seeded synthetic inputs for the benchmark configurations (host code).
//
// The reference's generators (util/random_string_generator.hpp) seed from
// std::random_device and so are not reproducible; these follow the same
// ideas — D/N-ratio strings (DNRatioGenerator :166-318), skewed lengths
// (SkewedDNRatioGenerator :431-509), suffixes of a text (SuffixGenerator
// :64-130) — with counter-based seeding so every string can be generated
// independently and in parallel.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/dsss.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {  // splitmix64 stream
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() { s += 0x9E3779B97F4A7C15ull; return splitmix64(s); }
    uint32_t below(uint32_t m) { return (uint32_t)(((next() >> 32) * (uint64_t)m) >> 32); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Bijection on [0, n): a 4-round Feistel network on the smallest even-width
// power-of-two domain >= n, with cycle walking back into [0, n).
struct FeistelPerm {
    uint64_t n;
    uint32_t half;
    uint64_t mask;
    uint64_t key[4];
    FeistelPerm(uint64_t n_, uint64_t seed) : n(n_) {
        uint32_t bits = 2;
        while (bits < 64 && (1ull << bits) < n) bits += 2;
        half = bits / 2;
        mask = (1ull << half) - 1;
        for (int r = 0; r < 4; ++r) key[r] = splitmix64(seed * 4 + r + 0x51ED);
    }
    uint64_t once(uint64_t x) const {
        uint64_t l = x >> half, r = x & mask;
        for (int k = 0; k < 4; ++k) {
            uint64_t f = splitmix64(r ^ key[k]) & mask;
            uint64_t nl = r;
            r = l ^ f;
            l = nl;
        }
        return (l << half) | r;
    }
    uint64_t operator()(uint64_t x) const {
        do { x = once(x); } while (x >= n);
        return x;
    }
};

template <typename F>
void parallel_for(uint64_t n, F&& f) {
    unsigned t = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 65536) t = 1;
    std::vector<std::thread> th;
    for (unsigned k = 0; k < t; ++k)
        th.emplace_back([&, k] {
            uint64_t b = n * k / t, e = n * (k + 1) / t;
            for (uint64_t i = b; i < e; ++i) f(i);
        });
    for (auto& x : th) x.join();
}

uint32_t digits26(uint64_t n) {
    uint32_t d = 1;
    unsigned __int128 v = 26;
    while (v < n) { v *= 26; ++d; }
    return d;
}

}  // namespace

extern "C" int dsss_gen_dn(uint64_t n, uint32_t len_short, uint32_t k_short, uint32_t len_long,
                           uint32_t k_long, double frac_long, uint64_t seed, uint8_t* chars,
                           uint64_t* offsets, uint32_t* lengths, uint64_t* char_bytes) {
    if (!char_bytes) return DSSS_EINVAL;
    const uint32_t d = digits26(n);
    if (k_short < d || k_short > len_short) return DSSS_EINVAL;
    if (frac_long > 0 && (k_long < d || k_long > len_long)) return DSSS_EINVAL;
    const uint64_t thr = frac_long <= 0 ? 0 : frac_long >= 1 ? UINT64_MAX
                                                          : (uint64_t)(frac_long * 18446744073709551616.0);
    const uint64_t cls_seed = splitmix64(seed ^ 0xC1A55ull);
    auto is_long = [&](uint64_t i) { return thr != 0 && splitmix64(cls_seed + i) < thr; };
    if (!chars) {
        uint64_t nl = 0;
        for (uint64_t i = 0; i < n; ++i) nl += is_long(i);
        *char_bytes = nl * (len_long + 1ull) + (n - nl) * (len_short + 1ull);
        return DSSS_OK;
    }
    if (!offsets || !lengths) return DSSS_EINVAL;
    uint64_t pos = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t L = is_long(i) ? len_long : len_short;
        offsets[i] = pos;
        lengths[i] = L;
        pos += L + 1ull;
    }
    *char_bytes = pos;
    FeistelPerm pi(n, seed);
    const uint64_t str_seed = splitmix64(seed ^ 0x5EEDull);
    parallel_for(n, [&](uint64_t i) {
        const bool lg = is_long(i);
        const uint32_t L = lg ? len_long : len_short, k = lg ? k_long : k_short;
        uint8_t* s = chars + offsets[i];
        std::memset(s, 'A', k - d);
        uint64_t v = pi(i);
        for (uint32_t j = 0; j < d; ++j) {
            s[k - 1 - j] = (uint8_t)('A' + v % 26);
            v /= 26;
        }
        Rng r(splitmix64(str_seed + i));
        for (uint32_t j = k; j < L; ++j) s[j] = (uint8_t)('A' + r.below(26));
        s[L] = 0;
    });
    return DSSS_OK;
}

extern "C" int dsss_gen_markov_text(uint64_t text_len, double copy_prob, uint64_t seed, uint8_t* text) {
    if (!text) return DSSS_EINVAL;
    static const uint8_t sym[4] = {'A', 'C', 'G', 'T'};
    Rng r(splitmix64(seed ^ 0x7E47ull));
    // 64 contexts (last three symbols) x 4 next-symbol weights.
    uint32_t cum[64][4];
    for (int c = 0; c < 64; ++c) {
        double w[4], tot = 0;
        for (int k = 0; k < 4; ++k) { w[k] = 0.05 + r.unit(); tot += w[k]; }
        double acc = 0;
        for (int k = 0; k < 4; ++k) {
            acc += w[k] / tot;
            cum[c][k] = k == 3 ? 0xFFFFFFFFu : (uint32_t)(acc * 4294967295.0);
        }
    }
    const uint64_t copy_thr = (uint64_t)(copy_prob * 18446744073709551616.0);
    uint32_t ctx = 0;
    std::vector<uint8_t> code(text_len);
    uint64_t pos = 0;
    while (pos < text_len) {
        if (pos > 0 && copy_prob > 0 && r.next() < copy_thr) {
            uint64_t len = 1024 + r.below(3073);
            uint64_t src = (uint64_t)(r.unit() * (double)pos);
            if (src >= pos) src = pos - 1;
            for (uint64_t j = 0; j < len && pos < text_len; ++j, ++pos) {
                code[pos] = code[src + j];  // may overlap the bytes being written, as LZ77 copies do
                ctx = ((ctx << 2) | code[pos]) & 63;
            }
            continue;
        }
        uint32_t u = (uint32_t)(r.next() >> 32);
        uint8_t k = 0;
        while (k < 3 && u > cum[ctx][k]) ++k;
        code[pos++] = k;
        ctx = ((ctx << 2) | k) & 63;
    }
    for (uint64_t i = 0; i < text_len; ++i) text[i] = sym[code[i]];
    return DSSS_OK;
}

extern "C" int dsss_gen_suffixes(uint64_t text_len, uint32_t max_len, uint64_t* offsets, uint32_t* lengths) {
    if (!offsets || !lengths) return DSSS_EINVAL;
    parallel_for(text_len, [&](uint64_t i) {
        offsets[i] = i;
        lengths[i] = (uint32_t)std::min<uint64_t>(max_len, text_len - i);
    });
    return DSSS_OK;
}

extern "C" int dsss_gen_request(uint64_t n, uint32_t min_len, uint32_t max_len, double zipf_s,
                                uint64_t seed, uint8_t* chars, uint64_t* offsets, uint32_t* lengths,
                                uint64_t* char_bytes) {
    if (!char_bytes || min_len == 0 || max_len < min_len) return DSSS_EINVAL;
    std::vector<double> cdf(max_len - min_len + 1);
    double acc = 0;
    for (uint32_t L = min_len; L <= max_len; ++L) {
        acc += std::pow((double)L, -zipf_s);
        cdf[L - min_len] = acc;
    }
    for (auto& c : cdf) c /= acc;
    const uint64_t len_seed = splitmix64(seed ^ 0x1E4Dull);
    auto length_of = [&](uint64_t i) {
        Rng r(splitmix64(len_seed + i));
        double u = r.unit();
        uint32_t k = (uint32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        return min_len + std::min<uint32_t>(k, max_len - min_len);
    };
    if (!chars) {
        uint64_t tot = 0;
        for (uint64_t i = 0; i < n; ++i) tot += length_of(i) + 1ull;
        *char_bytes = tot;
        return DSSS_OK;
    }
    if (!offsets || !lengths) return DSSS_EINVAL;
    uint64_t pos = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t L = length_of(i);
        offsets[i] = pos;
        lengths[i] = L;
        pos += L + 1ull;
    }
    *char_bytes = pos;
    std::vector<uint8_t> prefix(max_len / 2 + 1);
    Rng pr(splitmix64(seed ^ 0x9F1Full));
    for (auto& c : prefix) c = (uint8_t)(0x21 + pr.below(94));
    const uint64_t str_seed = splitmix64(seed ^ 0xB17Eull);
    parallel_for(n, [&](uint64_t i) {
        uint32_t L = lengths[i];
        uint8_t* s = chars + offsets[i];
        Rng r(splitmix64(str_seed + i));
        uint32_t pl = r.below(L / 2 + 1);
        std::memcpy(s, prefix.data(), pl);
        for (uint32_t j = pl; j < L; ++j) s[j] = (uint8_t)(0x21 + r.below(94));
        s[L] = 0;
    });
    return DSSS_OK;
}
