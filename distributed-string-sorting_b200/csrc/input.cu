// Input side: distribute_strings (src/mpi/readInput.hpp:40-104) for p PEs
// held by one GPU.  The reference gives rank r the r-th of p byte slices of
// the file (the first size % p slices one byte longer), turns every '\n' into
// a NUL, moves each rank's first line (up to and including its first '\n')
// to the previous rank, and ends the last rank's bytes with a NUL.  Together
// the ranks' vectors are the file with '\n' -> NUL, PE r > 0 starting just
// after the first '\n' of its slice, plus a NUL if the file does not end with
// one.  Here the boundaries come from one host search per slice, and the
// conversion, the line starts and the (offset, length) table are built on
// the device in two passes over 4096-byte tiles.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace dsss {

constexpr int LN_NT = 256, LN_BPT = 16, LN_TILE = LN_NT * LN_BPT;

__device__ __forceinline__ bool ln_term(uint32_t c) { return c == 0 || c == '\n'; }

// A thread's 16 bytes as one aligned load when the text is 16-byte aligned
// and the chunk lies inside it (full), and the byte before them: the
// previous lane's last byte by shuffle, lane 0's from memory (0 at position
// 0, where a line starts).  Every lane of the warp calls it.
__device__ __forceinline__ bool ln_chunk(const uint8_t* c, uint64_t S, uint64_t base, bool vec, uint32_t w[4],
                                         uint32_t& prev) {
    const bool full = vec && base + LN_BPT <= S;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (full) v = *reinterpret_cast<const uint4*>(c + base);
    w[0] = v.x;
    w[1] = v.y;
    w[2] = v.z;
    w[3] = v.w;
    prev = __shfl_up_sync(0xffffffffu, v.w >> 24, 1);
    if ((threadIdx.x & 31) == 0) prev = (base && base < S) ? c[base - 1] : 0u;
    return full;
}

// Pass 1: '\n' -> NUL, and the number of line starts per tile (position 0 and
// every position after a terminator).  A neighbour's byte read here is either
// the original '\n' or its NUL: both end a line.
__global__ void __launch_bounds__(LN_NT) k_lines_count(uint8_t* c, uint64_t S, uint32_t* tile_cnt) {
    __shared__ uint32_t part[LN_NT / 32];
    const uint64_t base = (uint64_t)blockIdx.x * LN_TILE + (uint64_t)threadIdx.x * LN_BPT;
    const bool vec = ((uintptr_t)c & 15) == 0;
    uint32_t cnt = 0, w[4], prev;
    if (ln_chunk(c, S, base, vec, w, prev)) {
        bool nl = false;
#pragma unroll
        for (int j = 0; j < LN_BPT; ++j) {
            const uint32_t v = (w[j >> 2] >> (8 * (j & 3))) & 0xFFu;
            cnt += ln_term(prev);
            prev = v;
            if (v == '\n') {
                w[j >> 2] &= ~(0xFFu << (8 * (j & 3)));
                nl = true;
            }
        }
        if (nl) *reinterpret_cast<uint4*>(c + base) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
#pragma unroll
        for (int j = 0; j < LN_BPT; ++j) {
            const uint64_t b = base + j;
            if (b >= S) break;
            const uint8_t v = c[b];
            if (b == 0 || ln_term(c[b - 1])) ++cnt;
            if (v == '\n') c[b] = 0;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < LN_NT / 32; ++w) t += part[w];
        tile_cnt[blockIdx.x] = t;
    }
}

// Pass 2: the offset of every line start, in order (tile_base: exclusive scan
// of pass 1's counts).
__global__ void __launch_bounds__(LN_NT) k_lines_offsets(const uint8_t* c, uint64_t S, const uint32_t* tile_base,
                                                         uint64_t* offsets) {
    __shared__ uint32_t wsum[LN_NT / 32];
    const uint64_t base = (uint64_t)blockIdx.x * LN_TILE + (uint64_t)threadIdx.x * LN_BPT;
    const bool vec = ((uintptr_t)c & 15) == 0;
    uint32_t mask = 0, wd[4], prev;
    if (ln_chunk(c, S, base, vec, wd, prev)) {
#pragma unroll
        for (int j = 0; j < LN_BPT; ++j) {
            if (prev == 0) mask |= 1u << j;
            prev = (wd[j >> 2] >> (8 * (j & 3))) & 0xFFu;
        }
    } else {
#pragma unroll
        for (int j = 0; j < LN_BPT; ++j) {
            const uint64_t b = base + j;
            if (b < S && (b == 0 || c[b - 1] == 0)) mask |= 1u << j;
        }
    }
    const uint32_t cnt = __popc(mask);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t pre = tile_base[blockIdx.x] + x - cnt;
    for (int k = 0; k < w; ++k) pre += wsum[k];
    while (mask) {
        const int j = __ffs(mask) - 1;
        mask &= mask - 1;
        offsets[pre++] = base + j;
    }
}

// Lines are back to back, each followed by exactly one NUL.
__global__ void k_lines_len(const uint64_t* offsets, uint64_t n, uint64_t bytes, uint32_t* lengths) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint64_t e = k + 1 < n ? offsets[k + 1] : bytes;
    lengths[k] = (uint32_t)(e - offsets[k] - 1);
}

// First line of every PE: the first line start at or after its byte boundary.
__global__ void k_lines_parts(const uint64_t* offsets, uint64_t n, const uint64_t* bound, uint32_t p, uint64_t* pb) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > p) return;
    const uint64_t B = bound[r];
    uint64_t lo = 0, hi = n;  // first k with offsets[k] >= B
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (offsets[mid] < B) lo = mid + 1;
        else hi = mid;
    }
    pb[r] = lo;
}

}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_distribute_lines(dsss_ctx* ctx, const uint8_t* file, uint64_t size, uint64_t max_size, uint32_t p,
                          uint8_t* chars, uint64_t chars_cap, uint64_t* offsets, uint32_t* lengths, uint64_t cap_n,
                          uint64_t* n_out, uint64_t* char_bytes, uint64_t* part_begin, dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (p == 0) return fail(DSSS_EINVAL, "p must be >= 1");
    if (!n_out || !char_bytes || !part_begin) return fail(DSSS_EINVAL, "output pointers missing");
    if (size && !file) return fail(DSSS_EINVAL, "file is NULL");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t S = max_size ? std::min(size, max_size) : size;
    // slices (readInput.hpp:57-69) and the boundary after each slice's first '\n'
    std::vector<uint64_t> bound(p + 1, 0);
    const uint64_t slice = S / p, larger = S % p;
    if (slice == 0)  // the last slice is empty: the reference reads result.back() of an empty vector
        return fail(DSSS_EINVAL, "the file has fewer bytes (%llu) than PEs (%u)", (unsigned long long)S, p);
    for (uint32_t r = 1; r < p; ++r) {
        const uint64_t len = slice + (r < larger ? 1 : 0);
        const uint64_t off = r < larger ? len * r : larger * (slice + 1) + (r - larger) * slice;
        const void* nl = len ? memchr(file + off, '\n', len) : nullptr;
        if (!nl)
            return fail(DSSS_EINVAL,
                        "slice %u of %u holds no newline (the reference reads past its buffer there): "
                        "use fewer PEs or a file with shorter lines", r, p);
        bound[r] = (uint64_t)((const uint8_t*)nl - file) + 1;
    }
    const bool close = S && file[S - 1] != '\n' && file[S - 1] != 0;
    const uint64_t bytes = S + (close ? 1 : 0);
    bound[p] = bytes;
    *char_bytes = bytes;
    if (!chars) return DSSS_OK;
    if (chars_cap < bytes + 32) return fail(DSSS_EINVAL, "chars_cap below char_bytes + 32 padding");
    const uint64_t tiles = (S + LN_TILE - 1) / LN_TILE;
    if (tiles >= (1ull << 31)) return fail(DSSS_ENOTSUP, "file too large");
    Carve sz(nullptr);
    auto plan = [&](Carve& c, uint32_t*& cnt, uint32_t*& base, uint32_t*& tot, void*& scan, uint64_t*& bd,
                    uint64_t*& pbd) {
        cnt = c.take<uint32_t>(tiles ? tiles : 1);
        base = c.take<uint32_t>(tiles ? tiles : 1);
        tot = c.take<uint32_t>(2);
        scan = c.take<unsigned char>(scan_scratch_bytes(tiles ? tiles : 1));
        bd = c.take<uint64_t>(p + 1);
        pbd = c.take<uint64_t>(p + 1);
    };
    uint32_t *cnt, *base, *tot;
    void* scan;
    uint64_t *bd, *pbd;
    plan(sz, cnt, base, tot, scan, bd, pbd);
    DSSS_TRY(ensure_ws(ctx, sz.used));
    DSSS_TRY(ensure_pin(ctx, 4096));
    Carve c(ctx->ws);
    plan(c, cnt, base, tot, scan, bd, pbd);
    if (S) DSSS_CUDA(cudaMemcpyAsync(chars, file, S, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemsetAsync(chars + S, 0, chars_cap - S, st));
    uint32_t* pin = (uint32_t*)ctx->pin;
    uint64_t n = 0;
    if (S) {
        DSSS_LAUNCH("k_lines_count", st, k_lines_count<<<(unsigned)tiles, LN_NT, 0, st>>>(chars, S, cnt));
        DSSS_TRY(exclusive_scan_u32(cnt, base, tiles, tot, scan, st));
        DSSS_CUDA(cudaMemcpyAsync(pin, tot, 4, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        n = pin[0];
    }
    *n_out = n;
    if (n > cap_n) return fail(DSSS_EINVAL, "the file holds %llu lines, more than cap_n = %llu", (unsigned long long)n,
                               (unsigned long long)cap_n);
    if (n && (!offsets || !lengths)) return fail(DSSS_EINVAL, "offsets / lengths missing");
    DSSS_CUDA(cudaMemcpyAsync(bd, bound.data(), (p + 1) * 8, cudaMemcpyHostToDevice, st));
    if (n) {
        DSSS_LAUNCH("k_lines_offsets", st, k_lines_offsets<<<(unsigned)tiles, LN_NT, 0, st>>>(chars, S, base, offsets));
        DSSS_LAUNCH("k_lines_len", st, k_lines_len<<<grid_for(n, 256), 256, 0, st>>>(offsets, n, bytes, lengths));
    }
    DSSS_LAUNCH("k_lines_parts", st, k_lines_parts<<<grid_for(p + 1, 128), 128, 0, st>>>(offsets, n, bd, p, pbd));
    DSSS_CUDA(cudaMemcpyAsync(part_begin, pbd, (p + 1) * 8, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    part_begin[p] = n;
    return DSSS_OK;
}

}  // extern "C"
