// Seeded benchmark inputs generated in device memory, so that a
// configuration's strings never cross PCIe (the role of the reference's
// generators, util/random_string_generator.hpp:167-318 and :432-509, which
// build every PE's strings in place).  Same rules and the same bytes as the
// host generators in gen.cpp: every byte is a function of the seed, its
// string's index and its position, so the device computes each output word
// on its own.
//   D/N strings  : lengths and offsets (the seeded long class scanned), then
//                  every 16-byte word of the arena from its strings' rules;
//   suffix views : offsets[i] = i, lengths[i] = min(max_len, text_len - i);
//   requests     : Zipf lengths by inverse CDF, offsets by a scan, then the
//                  bytes (shared prefix, then the string's own draws).
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace dsss {
namespace {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t sm64(uint64_t x) {
    x += GOLDEN;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// t-th draw (t = 0, 1, ...) of the splitmix64 stream whose state starts at s0.
__device__ __forceinline__ uint64_t draw(uint64_t s0, uint64_t t) { return sm64(s0 + (t + 1) * GOLDEN); }
__device__ __forceinline__ uint32_t below(uint64_t x, uint32_t m) {
    return (uint32_t)(((x >> 32) * (uint64_t)m) >> 32);
}

struct FeistelDev {
    uint64_t n, mask;
    uint32_t half;
    uint64_t key[4];
};

FeistelDev feistel(uint64_t n, uint64_t seed) {
    FeistelDev f;
    f.n = n;
    uint32_t bits = 2;
    while (bits < 64 && (1ull << bits) < n) bits += 2;
    f.half = bits / 2;
    f.mask = (1ull << f.half) - 1;
    for (int r = 0; r < 4; ++r) f.key[r] = sm64(seed * 4 + r + 0x51ED);
    return f;
}

__device__ __forceinline__ uint64_t feistel_map(const FeistelDev& f, uint64_t x) {
    do {
        uint64_t l = x >> f.half, r = x & f.mask;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t t = r;
            r = l ^ (sm64(r ^ f.key[k]) & f.mask);
            l = t;
        }
        x = (l << f.half) | r;
    } while (x >= f.n);
    return x;
}

struct DnRule {
    uint64_t n, thr, cls_seed, str_seed;
    uint32_t len_short, k_short, len_long, k_long, d;
    FeistelDev perm;
};

__device__ __forceinline__ bool dn_long(const DnRule& R, uint64_t i) {
    return R.thr != 0 && sm64(R.cls_seed + i) < R.thr;
}

__global__ void k_dn_len1(DnRule R, uint32_t* len1, unsigned long long* nlong) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool lg = false;
    if (i < R.n) {
        lg = dn_long(R, i);
        if (len1) len1[i] = (lg ? R.len_long : R.len_short) + 1u;
    }
    const unsigned b = __ballot_sync(0xffffffffu, lg);
    if ((threadIdx.x & 31) == 0 && b && nlong) atomicAdd(nlong, (unsigned long long)__popc(b));
}

// lengths from len + 1; fixed-length sets: offsets without a scan
__global__ void k_dn_lengths(DnRule R, const uint32_t* len1, uint64_t* offsets, uint32_t* lengths) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.n) return;
    if (len1) {
        lengths[i] = len1[i] - 1u;
    } else {
        lengths[i] = R.len_short;
        offsets[i] = i * (R.len_short + 1ull);
    }
}

// Byte j of string i (j <= its length; the last is the NUL).
__device__ __forceinline__ uint8_t dn_byte(const DnRule& R, uint64_t i, uint32_t j, bool lg, uint64_t v, uint64_t s0) {
    const uint32_t L = lg ? R.len_long : R.len_short, k = lg ? R.k_long : R.k_short;
    if (j >= L) return 0;
    if (j + R.d < k) return 'A';
    if (j < k) {
        uint32_t e = k - 1 - j;  // digit e of v, least significant first
        uint64_t x = v;
        for (uint32_t q = 0; q < e; ++q) x /= 26;
        return (uint8_t)('A' + x % 26);
    }
    return (uint8_t)('A' + below(draw(s0, j - k), 26));
}

// One thread per 16-byte word of the arena: the word's bytes from the
// strings they belong to (found by a search over the offsets).
__global__ void __launch_bounds__(256) k_dn_chars(DnRule R, const uint64_t* offsets, uint64_t char_bytes,
                                                  uint8_t* chars) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t x0 = w * 16;
    if (x0 >= char_bytes) return;
    // the string holding byte x0: last i with offsets[i] <= x0
    uint64_t lo = 0, hi = R.n;
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (offsets[mid] <= x0) lo = mid;
        else hi = mid;
    }
    uint64_t i = lo, off = offsets[i];
    bool lg = dn_long(R, i);
    uint64_t v = feistel_map(R.perm, i), s0 = sm64(R.str_seed + i);
    uint64_t end = off + (lg ? R.len_long : R.len_short) + 1;
    uint8_t b[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const uint64_t x = x0 + q;
        if (x >= char_bytes) {
            b[q] = 0;
            continue;
        }
        if (x >= end) {  // the next string
            ++i;
            off = end;
            lg = dn_long(R, i);
            v = feistel_map(R.perm, i);
            s0 = sm64(R.str_seed + i);
            end = off + (lg ? R.len_long : R.len_short) + 1;
        }
        b[q] = dn_byte(R, i, (uint32_t)(x - off), lg, v, s0);
    }
    uint4 o;
    o.x = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
    o.y = b[4] | (b[5] << 8) | (b[6] << 16) | ((uint32_t)b[7] << 24);
    o.z = b[8] | (b[9] << 8) | (b[10] << 16) | ((uint32_t)b[11] << 24);
    o.w = b[12] | (b[13] << 8) | (b[14] << 16) | ((uint32_t)b[15] << 24);
    if (x0 + 16 <= char_bytes) {
        reinterpret_cast<uint4*>(chars)[w] = o;
    } else {
        for (int q = 0; q < 16 && x0 + q < char_bytes; ++q) chars[x0 + q] = b[q];
    }
}

__global__ void k_suffix_views(uint64_t text_len, uint32_t max_len, uint64_t* offsets, uint32_t* lengths) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= text_len) return;
    offsets[i] = i;
    const uint64_t r = text_len - i;
    lengths[i] = (uint32_t)(r < max_len ? r : max_len);
}

struct ReqRule {
    uint64_t n, len_seed, str_seed;
    uint32_t min_len, max_len;
    const double* cdf;  // max_len - min_len + 1 entries
    const uint8_t* prefix;
};

__device__ __forceinline__ uint32_t req_length(const ReqRule& R, uint64_t i) {
    const uint64_t s0 = sm64(R.len_seed + i);
    const double u = (double)(draw(s0, 0) >> 11) * (1.0 / 9007199254740992.0);
    uint32_t lo = 0, hi = R.max_len - R.min_len + 1;  // first k with cdf[k] >= u
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (R.cdf[mid] < u) lo = mid + 1;
        else hi = mid;
    }
    return R.min_len + min(lo, R.max_len - R.min_len);
}

__global__ void k_req_len1(ReqRule R, uint32_t* len1) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < R.n) len1[i] = req_length(R, i) + 1u;
}

__global__ void k_sum_len1(const uint32_t* len1, uint64_t n, unsigned long long* total) {
    unsigned long long t = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        t += len1[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(total, t);
}

__global__ void k_req_lengths(uint64_t n, const uint32_t* len1, uint32_t* lengths) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lengths[i] = len1[i] - 1u;
}

// One thread per string (lengths are at most 256): the shared prefix, then
// the string's own draws (draw 0 picks the prefix length).
__global__ void k_req_chars(ReqRule R, const uint64_t* offsets, const uint32_t* lengths, uint8_t* chars) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.n) return;
    const uint32_t L = lengths[i];
    uint8_t* s = chars + offsets[i];
    const uint64_t s0 = sm64(R.str_seed + i);
    const uint32_t pl = below(draw(s0, 0), L / 2 + 1);
    for (uint32_t j = 0; j < pl; ++j) s[j] = R.prefix[j];
    for (uint32_t j = pl; j < L; ++j) s[j] = (uint8_t)(0x21 + below(draw(s0, 1 + j - pl), 94));
    s[L] = 0;
}

uint32_t digits26(uint64_t n) {
    uint32_t d = 1;
    unsigned __int128 v = 26;
    while (v < n) { v *= 26; ++d; }
    return d;
}

}  // namespace
}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_gen_dn_dev(dsss_ctx* ctx, uint64_t n, uint32_t len_short, uint32_t k_short, uint32_t len_long,
                    uint32_t k_long, double frac_long, uint64_t seed, uint8_t* chars, uint64_t* offsets,
                    uint32_t* lengths, uint64_t* char_bytes, dsss_stream_t stream) {
    if (!ctx || !char_bytes) return fail(DSSS_EINVAL, "ctx and char_bytes are required");
    if (n >= (1ull << 32)) return fail(DSSS_EINVAL, "n must be below 2^32");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    DnRule R;
    R.n = n;
    R.d = digits26(n);
    if (k_short < R.d || k_short > len_short) return fail(DSSS_EINVAL, "k_short out of range");
    if (frac_long > 0 && (k_long < R.d || k_long > len_long)) return fail(DSSS_EINVAL, "k_long out of range");
    R.len_short = len_short;
    R.k_short = k_short;
    R.len_long = len_long;
    R.k_long = k_long;
    R.thr = frac_long <= 0 ? 0 : frac_long >= 1 ? UINT64_MAX : (uint64_t)(frac_long * 18446744073709551616.0);
    R.cls_seed = sm64(seed ^ 0xC1A55ull);
    R.str_seed = sm64(seed ^ 0x5EEDull);
    R.perm = feistel(n ? n : 1, seed);
    const bool mixed = R.thr != 0;
    // scratch: long count (+ len + 1 per string and the scan's partials)
    Carve sz(nullptr);
    sz.take<unsigned long long>(2);
    if (mixed) {
        sz.take<uint32_t>(n ? n : 1);
        sz.take<unsigned char>(scan_scratch_bytes(n));
    }
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 64));
    Carve c(ctx->ws);
    unsigned long long* cnt = c.take<unsigned long long>(2);
    uint32_t* len1 = mixed ? c.take<uint32_t>(n ? n : 1) : nullptr;
    void* scan = mixed ? (void*)c.take<unsigned char>(scan_scratch_bytes(n)) : nullptr;
    uint64_t nlong = 0;
    if (mixed && n) {
        DSSS_CUDA(cudaMemsetAsync(cnt, 0, 16, st));
        DSSS_LAUNCH("k_dn_len1", st, k_dn_len1<<<grid_for(n, 256), 256, 0, st>>>(R, chars ? len1 : nullptr, cnt));
        DSSS_CUDA(cudaMemcpyAsync(ctx->pin, cnt, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        nlong = *(uint64_t*)ctx->pin;
    }
    const uint64_t total = nlong * (len_long + 1ull) + (n - nlong) * (len_short + 1ull);
    *char_bytes = total;
    if (!chars) return DSSS_OK;
    if (!offsets || !lengths) return fail(DSSS_EINVAL, "offsets and lengths are required");
    if (n == 0) return DSSS_OK;
    if (mixed) DSSS_TRY(exclusive_scan_u32_to_u64(len1, offsets, n, (uint64_t*)(cnt + 1), scan, st));
    DSSS_LAUNCH("k_dn_lengths", st, k_dn_lengths<<<grid_for(n, 256), 256, 0, st>>>(R, len1, offsets, lengths));
    DSSS_LAUNCH("k_dn_chars", st, k_dn_chars<<<grid_for((total + 15) / 16, 256), 256, 0, st>>>(R, offsets, total, chars));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

int dsss_gen_suffixes_dev(uint64_t text_len, uint32_t max_len, uint64_t* offsets, uint32_t* lengths,
                          dsss_stream_t stream) {
    if (!offsets || !lengths) return fail(DSSS_EINVAL, "offsets and lengths are required");
    if (text_len >= (1ull << 32)) return fail(DSSS_EINVAL, "text_len must be below 2^32");
    if (!text_len) return DSSS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    DSSS_LAUNCH("k_suffix_views", st,
                k_suffix_views<<<grid_for(text_len, 256), 256, 0, st>>>(text_len, max_len, offsets, lengths));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

int dsss_gen_request_dev(dsss_ctx* ctx, uint64_t n, uint32_t min_len, uint32_t max_len, double zipf_s,
                         uint64_t seed, uint8_t* chars, uint64_t* offsets, uint32_t* lengths, uint64_t* char_bytes,
                         dsss_stream_t stream) {
    if (!ctx || !char_bytes || min_len == 0 || max_len < min_len) return fail(DSSS_EINVAL, "bad request arguments");
    if (n >= (1ull << 32)) return fail(DSSS_EINVAL, "n must be below 2^32");
    ActiveCtx active(ctx);
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t span = max_len - min_len + 1;
    std::vector<double> cdf(span);
    double acc = 0;
    for (uint32_t L = min_len; L <= max_len; ++L) {
        acc += std::pow((double)L, -zipf_s);
        cdf[L - min_len] = acc;
    }
    for (auto& x : cdf) x /= acc;
    std::vector<uint8_t> prefix(max_len / 2 + 1);
    {
        uint64_t s = sm64(seed ^ 0x9F1Full);
        for (auto& ch : prefix) {
            s += GOLDEN;
            ch = (uint8_t)(0x21 + (uint32_t)(((sm64(s) >> 32) * 94ull) >> 32));
        }
    }
    Carve sz(nullptr);
    sz.take<double>(span);
    sz.take<uint8_t>(prefix.size());
    sz.take<uint64_t>(1);
    sz.take<uint32_t>(n ? n : 1);
    sz.take<unsigned char>(scan_scratch_bytes(n));
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 64));
    Carve c(ctx->ws);
    double* dcdf = c.take<double>(span);
    uint8_t* dpre = c.take<uint8_t>(prefix.size());
    uint64_t* tot = c.take<uint64_t>(1);
    uint32_t* len1 = c.take<uint32_t>(n ? n : 1);
    void* scan = c.take<unsigned char>(scan_scratch_bytes(n));
    DSSS_CUDA(cudaMemcpyAsync(dcdf, cdf.data(), span * sizeof(double), cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(dpre, prefix.data(), prefix.size(), cudaMemcpyHostToDevice, st));
    ReqRule R{n, sm64(seed ^ 0x1E4Dull), sm64(seed ^ 0xB17Eull), min_len, max_len, dcdf, dpre};
    if (n) DSSS_LAUNCH("k_req_len1", st, k_req_len1<<<grid_for(n, 256), 256, 0, st>>>(R, len1));
    if (!chars) {  // the total only
        DSSS_CUDA(cudaMemsetAsync(tot, 0, 8, st));
        if (n) DSSS_LAUNCH("k_sum_len1", st, k_sum_len1<<<std::min<uint64_t>(grid_for(n, 256), 1184), 256, 0, st>>>(
                                              len1, n, (unsigned long long*)tot));
        DSSS_CUDA(cudaMemcpyAsync(ctx->pin, tot, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        *char_bytes = *(uint64_t*)ctx->pin;
        return DSSS_OK;
    }
    uint64_t* offs = offsets;
    if (!offs) return fail(DSSS_EINVAL, "offsets and lengths are required");
    if (!lengths) return fail(DSSS_EINVAL, "offsets and lengths are required");
    DSSS_TRY(exclusive_scan_u32_to_u64(len1, offs, n, tot, scan, st));
    DSSS_CUDA(cudaMemcpyAsync(ctx->pin, tot, 8, cudaMemcpyDeviceToHost, st));
    if (n) {
        DSSS_LAUNCH("k_req_lengths", st, k_req_lengths<<<grid_for(n, 256), 256, 0, st>>>(n, len1, lengths));
        DSSS_LAUNCH("k_req_chars", st, k_req_chars<<<grid_for(n, 128), 128, 0, st>>>(R, offs, lengths, chars));
    }
    DSSS_CUDA(cudaStreamSynchronize(st));
    *char_bytes = *(uint64_t*)ctx->pin;
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

}  // extern "C"
