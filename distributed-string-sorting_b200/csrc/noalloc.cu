// dsss_adjacent_lcp_noalloc: the adjacent-LCP kernel pair of util.cu with its
// scratch (the counter and queue of pairs handed to whole warps) in a
// fixed-size array compiled into the library instead of memory allocated per
// call.  For callers that must not call cudaMalloc: code running inside
// another framework's memory pool (a raw cudaMalloc bypasses the pool's
// accounting and can fail once the pool holds the device's free memory), and
// latency-critical loops where the implicit device synchronisation of
// cudaMalloc/cudaFree would stall every other stream.
#include <cstdio>
#include <mutex>

#include "internal.cuh"
#include "util.cuh"

namespace dsss {

// Largest m one call accepts; the array holds a 256-byte header (the counter)
// and one queue slot per string, 16 MiB + 256 B on every GPU that loads the
// library, for as long as the process runs.
constexpr uint64_t NOALLOC_MAX_STRINGS = 1ull << 22;
constexpr uint64_t NOALLOC_HEADER_WORDS = 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_HEADER_WORDS + NOALLOC_MAX_STRINGS];

// Device address of g_noalloc_scratch per device, looked up on the first call
// made with that device current (host code cannot use the symbol itself).
constexpr int NOALLOC_MAX_DEVICES = 64;
static void* g_noalloc_addr[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(void** out) {
    int dev = 0;
    DSSS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(DSSS_ENOTSUP, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(DSSS_EDEVICE, "cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return DSSS_OK;
}

}  // namespace dsss

using namespace dsss;

extern "C" int dsss_adjacent_lcp_noalloc(const dsss_arena* in, const uint32_t* order, uint64_t m, uint32_t* lcp,
                                         dsss_stream_t stream) {
    DSSS_TRY(check_arena(in));
    if (m > NOALLOC_MAX_STRINGS)
        return fail(DSSS_EINVAL, "dsss_adjacent_lcp_noalloc takes at most %llu strings per call (got %llu)",
                    (unsigned long long)NOALLOC_MAX_STRINGS, (unsigned long long)m);
    if (m && (!order || !lcp)) return fail(DSSS_EINVAL, "order/lcp is NULL");
    void* base = nullptr;
    DSSS_TRY(noalloc_scratch(&base));
    uint32_t* nlong = (uint32_t*)base;  // zeroed by adjacent_lcp before its kernels run
    uint32_t* longq = nlong + NOALLOC_HEADER_WORDS;
    ArenaDev a{in->chars, in->offsets, in->lengths, in->n};
    return adjacent_lcp(a, order, m, lcp, longq, nlong, (cudaStream_t)stream);
}
