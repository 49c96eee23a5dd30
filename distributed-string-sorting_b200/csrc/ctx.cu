// Context, error reporting, scratch management and the device-wide scan.
#include <cstdarg>
#include <cstring>

#include "internal.cuh"

namespace dsss {

static thread_local char g_err[512] = "";
thread_local KernelTimes* g_times = nullptr;

cudaEvent_t KernelTimes::get() {
    if (pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
}

void KernelTimes::fold() {
    for (auto& p : pending) {
        float ms = 0;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            size_t k = 0;
            while (k < names.size() && names[k] != p.name) ++k;
            if (k == names.size()) {
                names.emplace_back(p.name);
                total_ms.push_back(0);
                launches.push_back(0);
            }
            total_ms[k] += ms;
            launches[k] += 1;
        }
        pool.push_back(p.a);
        pool.push_back(p.b);
    }
    pending.clear();
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

// ------------------------------------------------------------- tuning ----
struct KnobDef {
    const char* name;
    int64_t def, lo, hi;
};
static const KnobDef g_knob_defs[TUNE_COUNT] = {
    {"dp_filter_min", 1ll << 40, 0, 1ll << 40},
    {"dp_filter_bits", 16, 4, 64},
    {"sort_small_max", 4096, 2, 4096},
    {"sort_pivot", 1, 0, 1},
    {"dp_table", 2, 2, 8},
    {"sort_graph_max_n", 0, 0, 1ll << 32},
    {"merge_by_sort", 1, 0, 2},
    {"merge_extend_lanes", 0, 0, 32},
    {"dp_split", 0, 0, 1},
    {"copy_word", 16, 8, 16},
    {"dp_digest", 4, 0, 64},
    {"dp_check", 0, 0, 1},
    {"sort_split_min", 0, 0, 1ll << 32},
    {"sort_bits", 0, 0, 3},
    {"sort_seg_bits", 0, 0, 1},
};
static std::atomic<int64_t> g_knobs[TUNE_COUNT] = {{1ll << 40}, {16}, {4096}, {1}, {2}, {0}, {1}, {0}, {0}, {16}, {4},
                                                   {0}, {0}, {0}, {0}};

int64_t tune(TuneKnob k) { return g_knobs[k].load(std::memory_order_relaxed); }

static int knob_index(const char* name) {
    if (!name) return -1;
    for (int k = 0; k < TUNE_COUNT; ++k)
        if (!strcmp(name, g_knob_defs[k].name)) return k;
    return -1;
}

int ensure_ws(Ctx* c, uint64_t bytes) {
    if (bytes <= c->ws_cap) return DSSS_OK;
    if (c->fixed_ws)
        return fail(DSSS_ENOMEM, "scratch of %llu bytes exceeds the fixed block of %llu bytes",
                    (unsigned long long)bytes, (unsigned long long)c->ws_cap);
    if (c->budget && bytes > c->budget)
        return fail(DSSS_ENOMEM, "scratch of %llu bytes exceeds the context budget of %llu bytes",
                    (unsigned long long)bytes, (unsigned long long)c->budget);
    if (c->ws) {
        DSSS_CUDA(cudaDeviceSynchronize());
        DSSS_CUDA(cudaFree(c->ws));
        c->ws = nullptr;
        c->ws_cap = 0;
    }
    uint64_t want = bytes + bytes / 8;  // headroom so slightly larger calls reuse it
    if (c->budget && want > c->budget) want = bytes;
    cudaError_t e = cudaMalloc(&c->ws, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->ws = nullptr;
        return fail(DSSS_ENOMEM, "cudaMalloc of %llu scratch bytes failed: %s", (unsigned long long)want,
                    cudaGetErrorString(e));
    }
    c->ws_cap = want;
    return DSSS_OK;
}

int ensure_pin(Ctx* c, uint64_t bytes) {
    if (bytes <= c->pin_cap) return DSSS_OK;
    if (c->pin) {
        DSSS_CUDA(cudaFreeHost(c->pin));
        c->pin = nullptr;
        c->pin_cap = 0;
    }
    uint64_t want = bytes < 4096 ? 4096 : bytes * 2;
    DSSS_CUDA(cudaMallocHost(&c->pin, want));
    c->pin_cap = want;
    return DSSS_OK;
}

int check_arena(const dsss_arena* a) {
    if (!a) return fail(DSSS_EINVAL, "arena is NULL");
    if (a->n && (!a->chars || !a->offsets || !a->lengths))
        return fail(DSSS_EINVAL, "arena with n = %llu has a NULL array", (unsigned long long)a->n);
    if (a->n >= (1ull << 32)) return fail(DSSS_EINVAL, "n = %llu exceeds 2^32-1 strings", (unsigned long long)a->n);
    if (((uintptr_t)a->chars & 7) != 0) return fail(DSSS_EINVAL, "arena chars must be 8-byte aligned");
    return DSSS_OK;
}

// ----------------------------------------------------- exclusive scan u32 ----
// Three passes: per-tile sums, a single-CTA scan of the sums, per-tile scan.
constexpr int SCAN_NT = 512, SCAN_IPT = 8, SCAN_TILE = SCAN_NT * SCAN_IPT;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    uint32_t base = w ? sh[w - 1] : 0;
    if (total) *total = sh[nw - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void scan_tile_sums(const uint32_t* in, uint64_t n, uint32_t* sums) {
    __shared__ uint32_t sh[32];
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + (uint64_t)k * SCAN_NT + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t tot;
    block_excl_scan(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_sums(uint32_t* sums, uint64_t m, uint32_t* total) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (uint64_t b = 0; b < m; b += SCAN_NT) {
        uint64_t i = b + threadIdx.x;
        uint32_t v = i < m ? sums[i] : 0;
        uint32_t tot;
        uint32_t ex = block_excl_scan(v, sh, &tot);
        if (i < m) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n, const uint32_t* sums) {
    __shared__ uint32_t sh[32];
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_IPT;
    uint32_t v[SCAN_IPT];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    uint32_t ex = block_excl_scan(s, sh, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
}

uint64_t scan_scratch_bytes(uint64_t n) { return ((n + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(uint64_t); }

// 64-bit variant (values summed in u64).
__device__ __forceinline__ uint64_t block_excl_scan64(uint64_t v, uint64_t* sh, uint64_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint64_t s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    uint64_t base = w ? sh[w - 1] : 0;
    if (total) *total = sh[nw - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void scan64_tile_sums(const uint32_t* in, uint64_t n, uint64_t* sums) {
    __shared__ uint64_t sh[32];
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint64_t s = 0;
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + (uint64_t)k * SCAN_NT + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint64_t tot;
    block_excl_scan64(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan64_sums(uint64_t* sums, uint64_t m, uint64_t* total) {
    __shared__ uint64_t sh[32];
    uint64_t carry = 0;
    for (uint64_t b = 0; b < m; b += SCAN_NT) {
        uint64_t i = b + threadIdx.x;
        uint64_t v = i < m ? sums[i] : 0;
        uint64_t tot;
        uint64_t ex = block_excl_scan64(v, sh, &tot);
        if (i < m) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan64_tiles(const uint32_t* in, uint64_t* out, uint64_t n, const uint64_t* sums) {
    __shared__ uint64_t sh[32];
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_IPT;
    uint32_t v[SCAN_IPT];
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    uint64_t ex = block_excl_scan64(s, sh, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_IPT; ++k) {
        uint64_t i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
}

int exclusive_scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, uint64_t* total, void* scratch,
                              cudaStream_t st) {
    uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    uint64_t* sums = (uint64_t*)scratch;
    if (n == 0) {
        if (total) DSSS_CUDA(cudaMemsetAsync(total, 0, sizeof(uint64_t), st));
        return DSSS_OK;
    }
    DSSS_LAUNCH("scan64_tile_sums", st, scan64_tile_sums<<<(unsigned)tiles, SCAN_NT, 0, st>>>(in, n, sums));
    DSSS_LAUNCH("scan64_sums", st, scan64_sums<<<1, SCAN_NT, 0, st>>>(sums, tiles, total));
    DSSS_LAUNCH("scan64_tiles", st, scan64_tiles<<<(unsigned)tiles, SCAN_NT, 0, st>>>(in, out, n, sums));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, void* scratch,
                       cudaStream_t st) {
    uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    uint32_t* sums = (uint32_t*)scratch;
    if (n == 0) {
        if (total) DSSS_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), st));
        return DSSS_OK;
    }
    DSSS_LAUNCH("scan_tile_sums", st, scan_tile_sums<<<(unsigned)tiles, SCAN_NT, 0, st>>>(in, n, sums));
    DSSS_LAUNCH("scan_sums", st, scan_sums<<<1, SCAN_NT, 0, st>>>(sums, tiles, total));
    DSSS_LAUNCH("scan_tiles", st, scan_tiles<<<(unsigned)tiles, SCAN_NT, 0, st>>>(in, out, n, sums));
    DSSS_CUDA(cudaGetLastError());
    return DSSS_OK;
}

}  // namespace dsss

using namespace dsss;

extern "C" {

int dsss_ctx_create(int device, uint64_t hbm_budget_bytes, dsss_ctx** out) {
    if (!out) return fail(DSSS_EINVAL, "out is NULL");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(DSSS_EDEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) return fail(DSSS_EINVAL, "device %d out of range (%d devices)", device, count);
    DSSS_CUDA(cudaSetDevice(device));
    dsss_ctx* c = new dsss_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    *out = c;
    return DSSS_OK;
}

int dsss_ctx_set_timing(dsss_ctx* c, int on) {
    if (!c) return fail(DSSS_EINVAL, "ctx is NULL");
    if (!c->times) c->times = new KernelTimes();
    c->times->on = on != 0;
    if (on) {
        c->times->names.clear();
        c->times->total_ms.clear();
        c->times->launches.clear();
    }
    return DSSS_OK;
}

int dsss_ctx_kernel_times(dsss_ctx* c, char* buf, uint64_t len) {
    if (!c || !buf || !len) return fail(DSSS_EINVAL, "ctx/buf is NULL");
    buf[0] = 0;
    if (!c->times) return DSSS_OK;
    c->times->fold();
    uint64_t used = 0;
    for (size_t k = 0; k < c->times->names.size(); ++k) {
        int w = snprintf(buf + used, len - used, "%s %llu %.6f\n", c->times->names[k].c_str(),
                         (unsigned long long)c->times->launches[k], c->times->total_ms[k]);
        if (w < 0 || (uint64_t)w >= len - used) return fail(DSSS_EINVAL, "buffer too small");
        used += (uint64_t)w;
    }
    return DSSS_OK;
}

int dsss_ctx_destroy(dsss_ctx* c) {
    if (!c) return DSSS_OK;
    if (c->times) {
        c->times->fold();
        for (auto e : c->times->pool) cudaEventDestroy(e);
        delete c->times;
    }
    if (c->ws) cudaFree(c->ws);
    if (c->pin) cudaFreeHost(c->pin);
    delete c;
    return DSSS_OK;
}

uint64_t dsss_ctx_scratch_bytes(const dsss_ctx* c) { return c ? c->ws_cap : 0; }

const char* dsss_last_error(void) { return g_err; }

int dsss_abi_version(void) { return DSSS_ABI_VERSION; }

int dsss_tune_set(const char* name, int64_t value) {
    const int k = knob_index(name);
    if (k < 0) return fail(DSSS_EINVAL, "unknown tuning knob '%s'", name ? name : "(null)");
    if (value < 0) value = g_knob_defs[k].def;
    if (value < g_knob_defs[k].lo || value > g_knob_defs[k].hi)
        return fail(DSSS_EINVAL, "knob %s takes %lld..%lld", name, (long long)g_knob_defs[k].lo,
                    (long long)g_knob_defs[k].hi);
    if (k == TUNE_MERGE_LANES && value && (value < 4 || (value & (value - 1))))
        return fail(DSSS_EINVAL, "knob %s takes 0, 4, 8, 16 or 32", name);
    if (k == TUNE_COPY_WORD && value != 8 && value != 16) return fail(DSSS_EINVAL, "knob %s takes 8 or 16", name);
    g_knobs[k].store(value, std::memory_order_relaxed);
    return DSSS_OK;
}

int dsss_tune_get(const char* name, int64_t* value) {
    const int k = knob_index(name);
    if (k < 0 || !value) return fail(DSSS_EINVAL, "unknown tuning knob '%s'", name ? name : "(null)");
    *value = g_knobs[k].load(std::memory_order_relaxed);
    return DSSS_OK;
}

}  // extern "C"
