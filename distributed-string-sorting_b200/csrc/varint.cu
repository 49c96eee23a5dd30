// Varint coding of LCP arrays for the string exchange with compressLcps
// (sendLcps, src/mpi/alltoall.hpp:406-425): Writer::PutVarint
// (src/encoding/integer_compression.hpp:66-140) writes 7 bits per byte, least
// significant first, the high bit set on every byte but the last; ranges
// (one per destination) are encoded back to back (IntegerCompression::
// writeRanges, src/mpi/byte_encoder.hpp:31-53) and decoded the same way
// (readRanges, :63-77).  On the GPU both directions are data-parallel: the
// encoder scans the per-value sizes, the decoder scans the end-of-value flags.
#include <vector>

#include "internal.cuh"

namespace dsss {

__device__ __forceinline__ uint32_t varint_size(uint32_t v) {
    return v < (1u << 7) ? 1 : v < (1u << 14) ? 2 : v < (1u << 21) ? 3 : v < (1u << 28) ? 4 : 5;
}

__global__ void k_varint_sizes(const uint32_t* v, uint64_t n, uint32_t* sz) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sz[i] = varint_size(v[i]);
}

__global__ void k_varint_write(const uint32_t* v, uint64_t n, const uint64_t* at, uint8_t* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x = v[i];
    uint8_t* o = out + at[i];
    const uint32_t m = varint_size(x);
    for (uint32_t k = 0; k + 1 < m; ++k) {
        o[k] = (uint8_t)((x & 0x7Fu) | 0x80u);
        x >>= 7;
    }
    o[m - 1] = (uint8_t)(x & 0x7Fu);
}

// Byte offsets of the range boundaries (value indices) from the scanned sizes.
__global__ void k_varint_bounds(const uint64_t* at, uint64_t n, uint64_t total, const uint64_t* bound, uint32_t nb,
                                uint64_t* out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nb) out[r] = bound[r] < n ? at[bound[r]] : total;
}

__global__ void k_varint_ends(const uint8_t* in, uint64_t m, uint32_t* flag, uint32_t* err) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m) return;
    flag[b] = (in[b] & 0x80u) ? 0u : 1u;
    if (b == m - 1 && (in[b] & 0x80u)) atomicExch(err, 1u);  // the last value is cut off
}

__global__ void k_varint_end_pos(const uint32_t* flag, const uint32_t* idx, uint64_t m, uint64_t n, uint64_t* ends,
                                 uint32_t* err) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m || !flag[b]) return;
    if (idx[b] >= n) {
        atomicExch(err, 1u);
        return;
    }
    ends[idx[b]] = b;
}

__global__ void k_varint_read(const uint8_t* in, const uint64_t* ends, uint64_t n, uint32_t* v, uint32_t* err) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint64_t s = k ? ends[k - 1] + 1 : 0, e = ends[k];
    if (e < s || e - s >= 5) {  // more than 5 bytes: not a 32-bit value
        atomicExch(err, 1u);
        v[k] = 0;
        return;
    }
    uint64_t x = 0;
    for (uint64_t b = s; b <= e; ++b) x |= (uint64_t)(in[b] & 0x7Fu) << (7 * (b - s));
    if (x > 0xFFFFFFFFull) atomicExch(err, 1u);
    v[k] = (uint32_t)x;
}

}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_varint_encode(dsss_ctx* ctx, const uint32_t* values, uint64_t n, const uint64_t* range_begin,
                       uint32_t nranges, uint8_t* out, uint64_t out_cap, uint64_t* out_bytes, uint64_t* range_bytes,
                       dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if (!out_bytes || (nranges && (!range_begin || !range_bytes))) return fail(DSSS_EINVAL, "output pointers missing");
    if (n && !values) return fail(DSSS_EINVAL, "values is NULL");
    if (nranges && range_begin[0] != 0) return fail(DSSS_EINVAL, "range_begin must start at 0");
    for (uint32_t r = 0; r < nranges; ++r)
        if (range_begin[r] > range_begin[r + 1] || range_begin[r + 1] > n)
            return fail(DSSS_EINVAL, "range_begin must rise from 0 to at most n");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t N = n ? n : 1;
    auto plan = [&](Carve& c, uint32_t*& sz, uint64_t*& at, uint64_t*& tot, void*& scan, uint64_t*& bd,
                    uint64_t*& bo) {
        sz = c.take<uint32_t>(N);
        at = c.take<uint64_t>(N);
        tot = c.take<uint64_t>(1);
        scan = c.take<unsigned char>(scan_scratch_bytes(N));
        bd = c.take<uint64_t>(nranges + 1);
        bo = c.take<uint64_t>(nranges + 1);
    };
    uint32_t* sz;
    uint64_t *at, *tot, *bd, *bo;
    void* scan;
    Carve s0(nullptr);
    plan(s0, sz, at, tot, scan, bd, bo);
    DSSS_TRY(ensure_ws(ctx, s0.used));
    DSSS_TRY(ensure_pin(ctx, 8 * (nranges + 2)));
    Carve c(ctx->ws);
    plan(c, sz, at, tot, scan, bd, bo);
    uint64_t* pin = (uint64_t*)ctx->pin;
    uint64_t total = 0;
    if (n) {
        DSSS_LAUNCH("k_varint_sizes", st, k_varint_sizes<<<grid_for(n, 256), 256, 0, st>>>(values, n, sz));
        DSSS_TRY(exclusive_scan_u32_to_u64(sz, at, n, tot, scan, st));
        DSSS_CUDA(cudaMemcpyAsync(pin, tot, 8, cudaMemcpyDeviceToHost, st));
        DSSS_CUDA(cudaStreamSynchronize(st));
        total = pin[0];
    }
    *out_bytes = total;
    if (!out) return DSSS_OK;  // size query
    if (total > out_cap) return fail(DSSS_EINVAL, "out_cap %llu below the %llu encoded bytes",
                                     (unsigned long long)out_cap, (unsigned long long)total);
    if (n) DSSS_LAUNCH("k_varint_write", st, k_varint_write<<<grid_for(n, 256), 256, 0, st>>>(values, n, at, out));
    if (nranges) {
        DSSS_CUDA(cudaMemcpyAsync(bd, range_begin, (nranges + 1) * 8, cudaMemcpyHostToDevice, st));
        DSSS_LAUNCH("k_varint_bounds", st,
                    k_varint_bounds<<<grid_for(nranges + 1, 128), 128, 0, st>>>(at, n, total, bd, nranges + 1, bo));
        DSSS_CUDA(cudaMemcpyAsync(pin, bo, (nranges + 1) * 8, cudaMemcpyDeviceToHost, st));
    }
    DSSS_CUDA(cudaStreamSynchronize(st));
    for (uint32_t r = 0; r < nranges; ++r) range_bytes[r] = pin[r + 1] - pin[r];
    return DSSS_OK;
}

int dsss_varint_decode(dsss_ctx* ctx, const uint8_t* in, uint64_t nbytes, uint32_t* values, uint64_t n,
                       dsss_stream_t stream) {
    if (!ctx) return fail(DSSS_EINVAL, "ctx is NULL");
    ActiveCtx active(ctx);
    if ((nbytes && !in) || (n && !values)) return fail(DSSS_EINVAL, "buffers missing");
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (nbytes == 0) {
        if (n) return fail(DSSS_EINVAL, "no bytes for %llu values", (unsigned long long)n);
        return DSSS_OK;
    }
    if (nbytes >= (1ull << 32)) return fail(DSSS_ENOTSUP, "more than 4 GiB of coded values per call");
    auto plan = [&](Carve& c, uint32_t*& flag, uint32_t*& idx, uint32_t*& tot, void*& scan, uint64_t*& ends,
                    uint32_t*& err) {
        flag = c.take<uint32_t>(nbytes);
        idx = c.take<uint32_t>(nbytes);
        tot = c.take<uint32_t>(1);
        scan = c.take<unsigned char>(scan_scratch_bytes(nbytes));
        ends = c.take<uint64_t>(n ? n : 1);
        err = c.take<uint32_t>(1);
    };
    uint32_t *flag, *idx, *tot, *err;
    uint64_t* ends;
    void* scan;
    Carve s0(nullptr);
    plan(s0, flag, idx, tot, scan, ends, err);
    DSSS_TRY(ensure_ws(ctx, s0.used));
    DSSS_TRY(ensure_pin(ctx, 64));
    Carve c(ctx->ws);
    plan(c, flag, idx, tot, scan, ends, err);
    uint32_t* pin = (uint32_t*)ctx->pin;
    DSSS_CUDA(cudaMemsetAsync(err, 0, 4, st));
    DSSS_LAUNCH("k_varint_ends", st, k_varint_ends<<<grid_for(nbytes, 256), 256, 0, st>>>(in, nbytes, flag, err));
    DSSS_TRY(exclusive_scan_u32(flag, idx, nbytes, tot, scan, st));
    DSSS_LAUNCH("k_varint_end_pos", st,
                k_varint_end_pos<<<grid_for(nbytes, 256), 256, 0, st>>>(flag, idx, nbytes, n, ends, err));
    DSSS_CUDA(cudaMemcpyAsync(pin, tot, 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0] != n)
        return fail(DSSS_EINVAL, "the bytes hold %u values, not n = %llu", pin[0], (unsigned long long)n);
    if (n) DSSS_LAUNCH("k_varint_read", st, k_varint_read<<<grid_for(n, 256), 256, 0, st>>>(in, ends, n, values, err));
    DSSS_CUDA(cudaMemcpyAsync(pin, err, 4, cudaMemcpyDeviceToHost, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    if (pin[0]) return fail(DSSS_EINVAL, "a coded value is cut off, longer than 5 bytes or above 2^32 - 1");
    return DSSS_OK;
}

}  // extern "C"
