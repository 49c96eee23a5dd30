// ORACLE — test infrastructure only.
//
// A second, independent statement of the benchmark inputs' generation rules,
// so that the CPU reference arm and the tests can build the configurations'
// inputs without loading the product library, and so that the product's
// generators (host and device) are checked byte for byte against it.
//
// The rules (seeded, counter-based: every string depends only on the seed and
// its index):
//  * D/N strings: string i has length L (L_long for a seeded class of
//    frac_long of the strings), k - d filler 'A's, the d base-26 digits
//    ('A' = 0) of pi(i) where pi is a seeded Feistel bijection on [0, n) and
//    d = ceil(log26 n), then letters drawn from a splitmix64 stream seeded
//    per string.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

uint64_t sm64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Stream {
    uint64_t s;
    uint64_t next() { s += 0x9E3779B97F4A7C15ull; return sm64(s); }
    uint32_t below(uint32_t m) { return (uint32_t)(((next() >> 32) * (uint64_t)m) >> 32); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Feistel {
    uint64_t n, mask;
    uint32_t half;
    uint64_t key[4];
    Feistel(uint64_t n_, uint64_t seed) : n(n_) {
        uint32_t bits = 2;
        while (bits < 64 && (1ull << bits) < n) bits += 2;
        half = bits / 2;
        mask = (1ull << half) - 1;
        for (int r = 0; r < 4; ++r) key[r] = sm64(seed * 4 + r + 0x51ED);
    }
    uint64_t map(uint64_t x) const {
        do {
            uint64_t l = x >> half, r = x & mask;
            for (int k = 0; k < 4; ++k) {
                uint64_t t = r;
                r = l ^ (sm64(r ^ key[k]) & mask);
                l = t;
            }
            x = (l << half) | r;
        } while (x >= n);
        return x;
    }
};

uint32_t base26_digits(uint64_t n) {
    uint32_t d = 1;
    unsigned __int128 v = 26;
    while (v < n) { v *= 26; ++d; }
    return d;
}

}  // namespace

extern "C" {

// Same arguments and results as the product's dsss_gen_dn.
int oracle_gen_dn(uint64_t n, uint32_t len_short, uint32_t k_short, uint32_t len_long, uint32_t k_long,
                  double frac_long, uint64_t seed, uint8_t* chars, uint64_t* offsets, uint32_t* lengths,
                  uint64_t* char_bytes) {
    if (!char_bytes) return -22;
    const uint32_t d = base26_digits(n);
    if (k_short < d || k_short > len_short) return -22;
    if (frac_long > 0 && (k_long < d || k_long > len_long)) return -22;
    uint64_t thr = 0;
    if (frac_long >= 1) thr = UINT64_MAX;
    else if (frac_long > 0) thr = (uint64_t)(frac_long * 18446744073709551616.0);
    const uint64_t cls = sm64(seed ^ 0xC1A55ull);
    auto long_class = [&](uint64_t i) { return thr != 0 && sm64(cls + i) < thr; };
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t L = long_class(i) ? len_long : len_short;
        if (chars) {
            offsets[i] = total;
            lengths[i] = L;
        }
        total += L + 1ull;
    }
    *char_bytes = total;
    if (!chars) return 0;
    Feistel perm(n, seed);
    const uint64_t sseed = sm64(seed ^ 0x5EEDull);
    for (uint64_t i = 0; i < n; ++i) {
        const bool lg = long_class(i);
        const uint32_t L = lg ? len_long : len_short, k = lg ? k_long : k_short;
        uint8_t* s = chars + offsets[i];
        for (uint32_t j = 0; j + d < k; ++j) s[j] = 'A';
        uint64_t v = perm.map(i);
        for (uint32_t j = 0; j < d; ++j, v /= 26) s[k - 1 - j] = (uint8_t)('A' + v % 26);
        Stream r{sm64(sseed + i)};
        for (uint32_t j = k; j < L; ++j) s[j] = (uint8_t)('A' + r.below(26));
        s[L] = 0;
    }
    return 0;
}

}  // extern "C"
