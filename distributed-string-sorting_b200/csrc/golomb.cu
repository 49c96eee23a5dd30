// Golomb/delta coding of sorted 64-bit values: the wire format of the
// reference's hash exchange with sequentialGolombEncoding
// (AllToAllHashesGolomb, src/sorter/distributed/bloomfilter.hpp:164-313, over
// getDeltaEncoding / getDeltaDecoding, src/encoding/golomb_encoding.hpp:50-110,
// and thrill's Golomb bit streams, src/encoding/golomb_bit_stream.hpp,
// bit_stream.hpp, delta_stream.hpp).  A destination with c > 0 values gets
// the block [S, b, v_0, bit words], S the number of words after S; the bit
// words hold, most significant bit first, the code of every gap
// v_i - v_{i-1}: q = gap / b ones, a zero, and r = gap mod b in truncated
// binary (k = ceil(log2 b) bits holding r + 2^k - b when r >= 2^k - b, else
// k - 1 bits holding r); the last word's unused bits are ones.  A destination
// without values gets no words.
//
// Encoding is data-parallel: code lengths, a scan, then every code ORed into
// its words.  A variable-length code is read sequentially; the decoder cuts
// each block's bits into chunks of GB_CHUNK_BITS, reads every chunk from a
// guessed code start and repeats, each chunk then starting where its
// predecessor's last code ended, until no start changes.  The first chunk of
// a block starts right, so the starts are exact once they agree; Golomb
// codes fall back into step within a few codes, so nearly every guess holds
// after the first repetition (and after as many repetitions as a block has
// chunks in the worst case).
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace dsss {

constexpr uint64_t GB_CHUNK_BITS = 1024;
constexpr uint64_t GB_MAX_Q = 1ull << 31;  // longest unary part coded (a gap of 2^31 b)

static uint32_t gb_ceil_log2(uint64_t b) {  // tlx::integer_log2_ceil
    uint32_t k = 0;
    while (k < 64 && (1ull << k) < b) ++k;
    return k;
}

// Range of value i: the last r with rbeg[r] <= i (empty ranges share their
// start with the next range, which is the one that holds i).
__device__ __forceinline__ uint32_t gb_range_of(const uint64_t* rbeg, uint32_t nranges, uint64_t i) {
    uint32_t lo = 0, hi = nranges;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (rbeg[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

struct GbParams {
    const uint64_t* rbeg;  // nranges + 1 value indices
    const uint64_t* b;
    const uint64_t* little;  // 2^k - b
    const uint32_t* k;
    uint32_t nranges;
};

__device__ __forceinline__ void gb_code(const GbParams& P, uint32_t r, uint64_t gap, uint64_t& q, uint64_t& val,
                                        uint32_t& kk) {
    const uint64_t b = P.b[r], little = P.little[r];
    const uint32_t k = P.k[r];
    q = gap / b;
    const uint64_t rem = gap - q * b;
    if (rem >= little) {
        val = rem + little;
        kk = k;
    } else {
        val = rem;
        kk = k - 1;
    }
}

__global__ void k_gb_len(const uint64_t* v, uint64_t n, GbParams P, uint32_t* len, uint32_t* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = gb_range_of(P.rbeg, P.nranges, i);
    if (i == P.rbeg[r]) {  // the first value of a range is not coded
        len[i] = 0;
        return;
    }
    if (v[i] < v[i - 1]) atomicOr(err, 1u);  // not ascending
    uint64_t q, val;
    uint32_t kk;
    gb_code(P, r, v[i] - v[i - 1], q, val, kk);
    if (q > GB_MAX_Q) {
        atomicOr(err, 2u);
        len[i] = 0;
        return;
    }
    len[i] = (uint32_t)(q + 1 + kk);
}

// Bits and words of every range's block (0 words for an empty range).
__global__ void k_gb_range_words(const uint64_t* pos, uint64_t n, const uint64_t* total, GbParams P, uint64_t* rbits,
                                 uint64_t* rwords) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.nranges) return;
    const uint64_t b0 = P.rbeg[r], b1 = P.rbeg[r + 1];
    if (b1 == b0) {
        rbits[r] = 0;
        rwords[r] = 0;
        return;
    }
    const uint64_t bits = (b1 < n ? pos[b1] : *total) - pos[b0];
    rbits[r] = bits;
    rwords[r] = 3 + (bits + 63) / 64;
}

// Ones over bits [t, t + q) of w (bit 0 = the first word's most significant).
__device__ __forceinline__ void gb_ones(unsigned long long* w, uint64_t t, uint64_t q) {
    if (q == 0) return;
    const uint64_t e = t + q - 1;
    const uint64_t w0 = t >> 6, w1 = e >> 6;
    const uint32_t a = (uint32_t)(t & 63), z = (uint32_t)(e & 63);
    if (w0 == w1) {
        atomicOr(&w[w0], (~0ull >> a) & (~0ull << (63 - z)));
        return;
    }
    atomicOr(&w[w0], ~0ull >> a);
    for (uint64_t x = w0 + 1; x < w1; ++x) w[x] = ~0ull;  // words wholly inside one code
    atomicOr(&w[w1], ~0ull << (63 - z));
}

// The nb (1..64) low bits of val at bits [t, t + nb), most significant first.
__device__ __forceinline__ void gb_bits(unsigned long long* w, uint64_t t, uint64_t val, uint32_t nb) {
    const uint32_t a = (uint32_t)(t & 63);
    const uint64_t x = t >> 6;
    if (a + nb <= 64) {
        atomicOr(&w[x], (unsigned long long)(val << (64 - a - nb)));
    } else {
        const uint32_t second = a + nb - 64;
        atomicOr(&w[x], (unsigned long long)(val >> second));
        atomicOr(&w[x + 1], (unsigned long long)(val << (64 - second)));
    }
}

__global__ void k_gb_write(const uint64_t* v, uint64_t n, GbParams P, const uint64_t* pos, const uint64_t* woff,
                           unsigned long long* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = gb_range_of(P.rbeg, P.nranges, i);
    const uint64_t b0 = P.rbeg[r];
    if (i == b0) return;
    unsigned long long* w = out + woff[r] + 3;
    uint64_t t = pos[i] - pos[b0];
    uint64_t q, val;
    uint32_t kk;
    gb_code(P, r, v[i] - v[i - 1], q, val, kk);
    if (q > GB_MAX_Q) return;
    gb_ones(w, t, q);
    t += q + 1;  // the zero is already there
    if (kk) gb_bits(w, t, val, kk);
}

// Header words and the ones after the last code (after k_gb_write).
__global__ void k_gb_head(const uint64_t* v, GbParams P, const uint64_t* rbits, const uint64_t* rwords,
                          const uint64_t* woff, unsigned long long* out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.nranges || rwords[r] == 0) return;
    unsigned long long* w = out + woff[r];
    w[0] = rwords[r] - 1;
    w[1] = P.b[r];
    w[2] = v[P.rbeg[r]];
    const uint64_t bits = rbits[r];
    if (bits & 63) w[3 + bits / 64] |= ~0ull >> (bits & 63);
}

// ---------------------------------------------------------------- decode ----
// Block table: one thread follows the S words.  blk[4j..4j+3] = (position,
// S, b, first value) of block j; *nb the blocks; err bit 1: a block runs past the
// buffer, is too short or has b = 0; bit 2: more than max_blocks blocks.
__global__ void k_gb_blocks(const unsigned long long* w, uint64_t nwords, uint32_t max_blocks, uint64_t* blk,
                            uint32_t* nb, uint32_t* err) {
    uint64_t pos = 0;
    uint32_t j = 0;
    while (pos < nwords) {
        if (j >= max_blocks) {
            atomicOr(err, 2u);
            break;
        }
        const uint64_t S = w[pos];
        if (S < 2 || S > nwords - pos - 1 || w[pos + 1] == 0) {
            atomicOr(err, 1u);
            break;
        }
        blk[4 * j] = pos;
        blk[4 * j + 1] = S;
        blk[4 * j + 2] = w[pos + 1];
        blk[4 * j + 3] = w[pos + 2];
        ++j;
        pos += 1 + S;
    }
    *nb = j;
}

struct GbChunk {
    uint64_t cs, ce;     // the chunk's bits [cs, ce)
    uint64_t bit1;       // end of its block's bits
    uint64_t b, little;  // the block's parameters
    uint32_t k, blk;
};

// Bit t of the stream.
__device__ __forceinline__ uint32_t gb_bit(const unsigned long long* w, uint64_t t) {
    return (uint32_t)(w[t >> 6] >> (63 - (t & 63))) & 1u;
}

// Reads the code at t (t < bit1).  Returns false at the stream's end (only
// ones up to bit1: the padding); else sets the gap and moves t past the
// code (t > bit1: the code is cut off).
__device__ __forceinline__ bool gb_read(const unsigned long long* w, const GbChunk& C, uint64_t& t, uint64_t& gap) {
    uint64_t q = 0;
    for (;;) {  // ones up to the next zero, a word at a time
        const uint32_t a = (uint32_t)(t & 63);
        const uint64_t x = (uint64_t)w[t >> 6] << a;  // bits from t at the top
        const uint32_t avail = 64 - a;
        uint32_t ones = (uint32_t)__clzll(~x);  // leading ones (64 when all are)
        if (ones > avail) ones = avail;
        if (t + ones >= C.bit1) return false;  // no zero before the end
        t += ones;
        q += ones;
        if (ones < avail) break;  // the zero is at t
    }
    ++t;  // the zero
    uint64_t r = 0;
    if (C.k) {
        const uint32_t lo = C.k - 1;
        for (uint32_t j = 0; j < lo; ++j) r = (r << 1) | (t < C.bit1 ? gb_bit(w, t++) : (++t, 0u));
        if (r >= C.little) r = ((r << 1) | (t < C.bit1 ? gb_bit(w, t++) : (++t, 0u))) - C.little;
    }
    gap = q * C.b + r;
    return true;
}

// One reading of every chunk from its start g[c]: cnt[c] codes start in
// [g[c], ce), e[c] where the next code starts (bit1 at the stream's end).
__global__ void k_gb_walk(const unsigned long long* w, const GbChunk* ch, uint64_t nch, const uint64_t* g, uint64_t* e,
                          uint32_t* cnt, uint32_t* err) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    const GbChunk C = ch[c];
    uint64_t t = g[c];
    uint32_t m = 0;
    while (t < C.ce) {
        uint64_t gap;
        if (!gb_read(w, C, t, gap)) {
            t = C.bit1;
            break;
        }
        ++m;
    }
    if (t > C.bit1) atomicOr(err, 4u);  // a code cut off by the block's end
    e[c] = t;
    cnt[c] = m;
}

// Each chunk starts where its predecessor in the block stopped.
__global__ void k_gb_follow(const GbChunk* ch, uint64_t nch, const uint64_t* e, uint64_t* g, uint32_t* changed) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0 || c >= nch || ch[c].blk != ch[c - 1].blk) return;
    const uint64_t s = e[c - 1];
    if (s != g[c]) {
        g[c] = s;
        *changed = 1;
    }
}

// The values: chunk c's codes go to out[oc[c]..], each its block's first
// value plus the gaps up to it (base[c] = that sum before the chunk).
__global__ void k_gb_gaps(const unsigned long long* w, const GbChunk* ch, uint64_t nch, const uint64_t* g,
                          const uint64_t* oc, unsigned long long* out, unsigned long long* csum) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    const GbChunk C = ch[c];
    uint64_t t = g[c], o = oc[c], s = 0;
    while (t < C.ce) {
        uint64_t gap;
        if (!gb_read(w, C, t, gap)) break;
        s += gap;
        out[o++] = gap;
    }
    csum[c] = s;
}

// The blocks' uncoded first values: out[at[j]] = first[j].
__global__ void k_gb_firsts(const uint64_t* at, const uint64_t* first, uint32_t nb, unsigned long long* out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nb) out[at[j]] = first[j];
}

__global__ void k_gb_sums(const GbChunk* ch, uint64_t nch, const uint64_t* oc, const uint32_t* cnt,
                          const unsigned long long* base, unsigned long long* out) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    uint64_t run = base[c];
    const uint64_t o = oc[c];
    for (uint32_t j = 0; j < cnt[c]; ++j) {
        run += out[o + j];
        out[o + j] = run;
    }
}

}  // namespace dsss

using namespace dsss;

extern "C" {

uint64_t dsss_golomb_param(uint64_t max_value, uint64_t count) {
    if (count == 0) return 1;
    const uint64_t avg = max_value / count;
    if (avg < 1) return 1;
    const uint64_t k = (uint64_t)std::floor(std::log2((double)avg));
    return 1ull << k;
}

uint64_t dsss_golomb_param_hashes(uint64_t count, uint32_t p) {
    if (p == 0) return 0;
    const uint64_t b = dsss_golomb_param(~0ull / p, count);
    return b == 1 ? 20000000000ull : b;
}

int dsss_golomb_encode(dsss_ctx* ctx, const uint64_t* values, const uint64_t* range_counts, uint32_t nranges,
                       const uint64_t* b, uint64_t* out, uint64_t out_cap, uint64_t* out_words, uint64_t* range_words,
                       dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (!out_words || (nranges && (!range_counts || !b || !range_words)))
        return fail(DSSS_EINVAL, "output pointers missing");
    std::vector<uint64_t> rbeg(nranges + 1, 0), little(nranges), bb(nranges);
    std::vector<uint32_t> kk(nranges);
    for (uint32_t r = 0; r < nranges; ++r) {
        if (b[r] == 0) return fail(DSSS_EINVAL, "range %u: the Golomb parameter b must be >= 1", r);
        rbeg[r + 1] = rbeg[r] + range_counts[r];
        bb[r] = b[r];
        kk[r] = gb_ceil_log2(b[r]);
        little[r] = (kk[r] >= 64 ? 0ull : (1ull << kk[r])) - b[r];
    }
    const uint64_t n = rbeg[nranges];
    if (n && !values) return fail(DSSS_EINVAL, "values is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t N = n ? n : 1, R = nranges ? nranges : 1;
    auto plan = [&](Carve& c, uint32_t*& len, uint64_t*& pos, uint64_t*& tot, void*& scan, uint64_t*& prm,
                    uint32_t*& pk, uint64_t*& rbits, uint64_t*& rw, uint64_t*& woff, uint32_t*& err) {
        len = c.take<uint32_t>(N);
        pos = c.take<uint64_t>(N);
        tot = c.take<uint64_t>(1);
        scan = c.take<unsigned char>(scan_scratch_bytes(N));
        prm = c.take<uint64_t>(3 * R + 1);  // rbeg, b, little
        pk = c.take<uint32_t>(R);
        rbits = c.take<uint64_t>(R);
        rw = c.take<uint64_t>(R);
        woff = c.take<uint64_t>(R);
        err = c.take<uint32_t>(1);
    };
    uint32_t *len, *pk, *err;
    uint64_t *pos, *tot, *prm, *rbits, *rw, *woff;
    void* scan;
    Carve s0(nullptr);
    plan(s0, len, pos, tot, scan, prm, pk, rbits, rw, woff, err);
    DSSS_TRY(ensure_ws(ctx, s0.used));
    DSSS_TRY(ensure_pin(ctx, 8 * (R + 4)));
    Carve c(ctx->ws);
    plan(c, len, pos, tot, scan, prm, pk, rbits, rw, woff, err);
    uint64_t* pin = (uint64_t*)ctx->pin;
    *out_words = 0;
    if (nranges == 0) return DSSS_OK;
    DSSS_CUDA(cudaMemcpyAsync(prm, rbeg.data(), (nranges + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(prm + nranges + 1, bb.data(), nranges * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(prm + 2 * nranges + 1, little.data(), nranges * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(pk, kk.data(), nranges * 4, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemsetAsync(err, 0, 4, st));
    GbParams P{prm, prm + nranges + 1, prm + 2 * nranges + 1, pk, nranges};
    if (n) {
        DSSS_LAUNCH("k_gb_len", st, k_gb_len<<<grid_for(n, 256), 256, 0, st>>>(values, n, P, len, err));
        DSSS_TRY(exclusive_scan_u32_to_u64(len, pos, n, tot, scan, st));
    } else {
        DSSS_CUDA(cudaMemsetAsync(tot, 0, 8, st));
    }
    DSSS_LAUNCH("k_gb_range_words", st,
                k_gb_range_words<<<grid_for(nranges, 128), 128, 0, st>>>(pos, n, tot, P, rbits, rw));
    DSSS_CUDA(cudaMemcpyAsync(pin, rw, nranges * 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaMemcpyAsync(pin + nranges, err, 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    const uint32_t e = (uint32_t)(pin[nranges] & 0xFFFFFFFFu);
    if (e & 1u) return fail(DSSS_EINVAL, "the values of a range must be ascending");
    if (e & 2u) return fail(DSSS_EINVAL, "a gap needs more than 2^31 unary bits (b too small for the values)");
    std::vector<uint64_t> wo(nranges);
    uint64_t total = 0;
    for (uint32_t r = 0; r < nranges; ++r) {
        range_words[r] = pin[r];
        wo[r] = total;
        total += pin[r];
    }
    *out_words = total;
    if (!out) return DSSS_OK;  // size query
    if (total > out_cap) return fail(DSSS_EINVAL, "out_cap %llu below the %llu coded words",
                                     (unsigned long long)out_cap, (unsigned long long)total);
    if (total == 0) return DSSS_OK;
    DSSS_CUDA(cudaMemcpyAsync(woff, wo.data(), nranges * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemsetAsync(out, 0, total * 8, st));
    unsigned long long* o = (unsigned long long*)out;
    if (n) DSSS_LAUNCH("k_gb_write", st, k_gb_write<<<grid_for(n, 256), 256, 0, st>>>(values, n, P, pos, woff, o));
    DSSS_LAUNCH("k_gb_head", st, k_gb_head<<<grid_for(nranges, 128), 128, 0, st>>>(values, P, rbits, rw, woff, o));
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

int dsss_golomb_decode(dsss_ctx* ctx, const uint64_t* words, uint64_t nwords, uint64_t* values, uint64_t cap_values,
                       uint64_t* n_values, uint64_t* block_counts, uint32_t max_blocks, uint32_t* nblocks,
                       dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (!n_values || !nblocks || (max_blocks && !block_counts)) return fail(DSSS_EINVAL, "output pointers missing");
    if (nwords && !words) return fail(DSSS_EINVAL, "words is NULL");
    *n_values = 0;
    *nblocks = 0;
    if (nwords == 0) return DSSS_OK;
    if (max_blocks == 0) return fail(DSSS_EINVAL, "max_blocks is 0 for a non-empty buffer");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned long long* w = (const unsigned long long*)words;
    // 1. the block table
    {
        Carve s0(nullptr);
        s0.take<uint64_t>(4ull * max_blocks);
        s0.take<uint32_t>(2);
        DSSS_TRY(ensure_ws(ctx, s0.used));
    }
    DSSS_TRY(ensure_pin(ctx, 32ull * max_blocks + 64));
    std::vector<uint64_t> blk;
    uint32_t nb = 0;
    {
        Carve c(ctx->ws);
        uint64_t* dblk = c.take<uint64_t>(4ull * max_blocks);
        uint32_t* dnb = c.take<uint32_t>(2);
        DSSS_CUDA(cudaMemsetAsync(dnb, 0, 8, st));
        DSSS_LAUNCH("k_gb_blocks", st, k_gb_blocks<<<1, 1, 0, st>>>(w, nwords, max_blocks, dblk, dnb, dnb + 1));
        uint32_t* pin = (uint32_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin, dnb, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        nb = pin[0];
        if (pin[1] & 1u) return fail(DSSS_EINVAL, "a Golomb block runs past the buffer, is too short or has b = 0");
        if (pin[1] & 2u) return fail(DSSS_EINVAL, "more than max_blocks = %u blocks", max_blocks);
        blk.resize(4ull * nb);
        uint64_t* pin64 = (uint64_t*)ctx->pin;
        DSSS_CUDA(cudaMemcpyAsync(pin64, dblk, 32ull * nb, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        std::copy(pin64, pin64 + 4ull * nb, blk.begin());
    }
    // 2. chunks of every block's bits
    std::vector<GbChunk> ch;
    std::vector<uint64_t> g0;
    std::vector<uint64_t> first_chunk(nb + 1);
    for (uint32_t j = 0; j < nb; ++j) {
        const uint64_t pos = blk[4 * j], S = blk[4 * j + 1], b = blk[4 * j + 2];
        const uint32_t k = gb_ceil_log2(b);
        const uint64_t little = (k >= 64 ? 0ull : (1ull << k)) - b;
        const uint64_t bit0 = (pos + 3) * 64, bit1 = (pos + 1 + S) * 64;
        first_chunk[j] = ch.size();
        for (uint64_t cs = bit0; cs < bit1; cs += GB_CHUNK_BITS) {
            ch.push_back(GbChunk{cs, std::min(cs + GB_CHUNK_BITS, bit1), bit1, b, little, k, j});
            g0.push_back(cs);
        }
    }
    first_chunk[nb] = ch.size();
    const uint64_t nch = ch.size();
    const uint64_t NC = nch ? nch : 1;
    const uint64_t NB = nb ? nb : 1;
    auto plan = [&](Carve& c, GbChunk*& dch, uint64_t*& g, uint64_t*& e, uint32_t*& cnt, uint64_t*& oc,
                    unsigned long long*& csum, unsigned long long*& base, uint32_t*& flags, uint64_t*& fat) {
        dch = c.take<GbChunk>(NC);
        g = c.take<uint64_t>(NC);
        e = c.take<uint64_t>(NC);
        cnt = c.take<uint32_t>(NC);
        oc = c.take<uint64_t>(NC);
        csum = c.take<unsigned long long>(NC);
        base = c.take<unsigned long long>(NC);
        flags = c.take<uint32_t>(2);
        fat = c.take<uint64_t>(2 * NB);  // (output place, value) of every block's first value
    };
    GbChunk* dch;
    uint64_t *g, *e, *oc, *fat;
    uint32_t *cnt, *flags;
    unsigned long long *csum, *base;
    Carve s1(nullptr);
    plan(s1, dch, g, e, cnt, oc, csum, base, flags, fat);
    DSSS_TRY(ensure_ws(ctx, s1.used));
    DSSS_TRY(ensure_pin(ctx, 16 * NC + 64));
    Carve c(ctx->ws);
    plan(c, dch, g, e, cnt, oc, csum, base, flags, fat);
    std::vector<uint32_t> hcnt(nch);
    if (nch) {
        DSSS_CUDA(cudaMemcpyAsync(dch, ch.data(), nch * sizeof(GbChunk), cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaMemcpyAsync(g, g0.data(), nch * 8, cudaMemcpyHostToDevice, st));
        DSSS_CUDA(cudaStreamSynchronize(st));  // the host vectors are reused below
        uint32_t* pin = (uint32_t*)ctx->pin;
        // 3. read every chunk until the starts agree (at most one round per
        // chunk of the longest block, plus one)
        uint64_t longest = 0;
        for (uint32_t j = 0; j < nb; ++j) longest = std::max(longest, first_chunk[j + 1] - first_chunk[j]);
        bool settled = false;
        for (uint64_t round = 0; round <= longest && !settled; ++round) {
            DSSS_CUDA(cudaMemsetAsync(flags, 0, 8, st));
            DSSS_LAUNCH("k_gb_walk", st, k_gb_walk<<<grid_for(nch, 128), 128, 0, st>>>(w, dch, nch, g, e, cnt,
                                                                                       flags + 1));
            DSSS_LAUNCH("k_gb_follow", st, k_gb_follow<<<grid_for(nch, 256), 256, 0, st>>>(dch, nch, e, g, flags));
            DSSS_CUDA(cudaMemcpyAsync(pin, flags, 8, cudaMemcpyDeviceToHost, st));
            DSSS_CUDA(cudaStreamSynchronize(st));
            settled = pin[0] == 0;
            if (settled && (pin[1] & 4u)) return fail(DSSS_EINVAL, "a Golomb code is cut off by its block's end");
        }
        if (!settled) return fail(DSSS_EDEVICE, "Golomb chunk starts did not settle");
        DSSS_CUDA(cudaMemcpyAsync(pin, cnt, nch * 4, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        std::copy(pin, pin + nch, hcnt.begin());
    }
    // 4. output places: each block's first value, then its chunks' codes
    std::vector<uint64_t> hoc(nch), first_at(nb);
    uint64_t total = 0;
    for (uint32_t j = 0; j < nb; ++j) {
        first_at[j] = total++;
        uint64_t m = 0;
        for (uint64_t x = first_chunk[j]; x < first_chunk[j + 1]; ++x) {
            hoc[x] = total;
            total += hcnt[x];
            m += hcnt[x];
        }
        if (j < max_blocks) block_counts[j] = m + 1;
    }
    *n_values = total;
    *nblocks = nb;
    if (!values) return DSSS_OK;  // size query
    if (total > cap_values) return fail(DSSS_EINVAL, "cap_values %llu below the %llu coded values",
                                        (unsigned long long)cap_values, (unsigned long long)total);
    unsigned long long* out = (unsigned long long*)values;
    {  // the uncoded first values
        std::vector<uint64_t> fa(2ull * nb);
        for (uint32_t j = 0; j < nb; ++j) {
            fa[j] = first_at[j];
            fa[nb + j] = blk[4 * j + 3];
        }
        DSSS_CUDA(cudaMemcpyAsync(fat, fa.data(), 16ull * nb, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_gb_firsts", st, k_gb_firsts<<<grid_for(nb, 128), 128, 0, st>>>(fat, fat + nb, nb, out));
        DSSS_CUDA(cudaStreamSynchronize(st));  // fa is released below
    }
    if (nch) {
        DSSS_CUDA(cudaMemcpyAsync(oc, hoc.data(), nch * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_gb_gaps", st, k_gb_gaps<<<grid_for(nch, 128), 128, 0, st>>>(w, dch, nch, g, oc, out, csum));
        // each chunk's start: its block's first value plus the gaps before it
        uint64_t* pin64 = (uint64_t*)ctx->pin;
        std::vector<uint64_t> hs(nch), hb(nch);
        DSSS_CUDA(cudaMemcpyAsync(pin64, csum, nch * 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        std::copy(pin64, pin64 + nch, hs.begin());
        for (uint32_t j = 0; j < nb; ++j) {
            uint64_t run = blk[4 * j + 3];
            for (uint64_t x = first_chunk[j]; x < first_chunk[j + 1]; ++x) {
                hb[x] = run;
                run += hs[x];
            }
        }
        DSSS_CUDA(cudaMemcpyAsync(base, hb.data(), nch * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_gb_sums", st, k_gb_sums<<<grid_for(nch, 128), 128, 0, st>>>(dch, nch, oc, cnt, base, out));
    }
    DSSS_CUDA(cudaGetLastError());
    DSSS_CUDA(cudaStreamSynchronize(st));
    return DSSS_OK;
}

}  // extern "C"
