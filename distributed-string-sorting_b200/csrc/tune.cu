// Autotuner: times the full path on the caller's input under every setting of
// the tuning knobs in a small grid (small-segment cutoff of the string sort,
// pivot passes, the MSD digit: one key byte, sampled splitters where a key
// byte splits poorly, the keys' top differing bits in the passes over the
// arena or inside the segment sorter) and leaves the fastest setting in
// force.
// Results never depend on the knobs, so tuning only changes speed.  The
// digit's bucket count (256) and the scatter tile (2048 strings) are fixed in
// this build: the shared-memory histograms and the 13-byte-per-string
// staging of the scatter are sized for them.
#include <cstdio>
#include <vector>

#include "internal.cuh"
#include "pd.cuh"

using namespace dsss;

namespace {

constexpr int NKNOBS = 5;

struct Setting {
    int64_t small_max, pivot, split_min, bits, seg_bits;
};

struct Knobs {
    int64_t v[NKNOBS];
};

const char* const kNames[NKNOBS] = {"sort_small_max", "sort_pivot", "sort_split_min", "sort_bits", "sort_seg_bits"};

Knobs get_knobs() {
    Knobs k;
    for (int i = 0; i < NKNOBS; ++i) dsss_tune_get(kNames[i], &k.v[i]);
    return k;
}

void set_knobs(const int64_t* v) {
    for (int i = 0; i < NKNOBS; ++i) dsss_tune_set(kNames[i], v[i]);
}

}  // namespace

extern "C" int dsss_autotune(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p,
                             const uint64_t* part_begin, const dsss_opts* opts, uint32_t trials, dsss_tuning* out,
                             dsss_stream_t stream) {
    if (!ctx || !out) return fail(DSSS_EINVAL, "ctx/out is NULL");
    DSSS_TRY(check_arena(in));
    if (nsets == 0 || p == 0 || !part_begin) return fail(DSSS_EINVAL, "nsets/p/part_begin missing");
    if (trials == 0) trials = 2;
    DSSS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t n = in->n, N = n ? n : 1;
    const uint64_t npe = (uint64_t)nsets * p;
    // outputs of the trial runs (tuning is not on the hot path: plain allocations)
    uint32_t* dev = nullptr;
    DSSS_CUDA(cudaMalloc(&dev, 5 * N * sizeof(uint32_t)));
    std::vector<uint64_t> intervals(npe * p), recv(npe);
    dsss_pd_result r{dev, nullptr, dev + N, intervals.data(), dev + 2 * N, dev + 3 * N, dev + 4 * N, recv.data()};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const Knobs saved = get_knobs();
    Setting grid[5 * 3 * 2];
    {
        const int64_t smalls[3] = {4096, 1024, 256};
        // (split_min, bits, seg_bits)
        const int64_t digits[5][3] = {{0, 0, 0}, {65536, 0, 0}, {0, 2, 0}, {0, 0, 1}, {0, 3, 1}};
        int g = 0;
        for (int dgt = 0; dgt < 5; ++dgt)
            for (int pv = 1; pv >= 0; --pv)
                for (int sm = 0; sm < 3; ++sm)
                    grid[g++] = {smalls[sm], pv, digits[dgt][0], digits[dgt][1], digits[dgt][2]};
    }
    double best = 1e300, first = 0;
    int best_i = -1, rc = DSSS_OK;
    uint32_t tried = 0;
    for (int i = 0; i < (int)(sizeof grid / sizeof grid[0]) && rc == DSSS_OK; ++i) {
        const int64_t v[NKNOBS] = {grid[i].small_max, grid[i].pivot, grid[i].split_min, grid[i].bits,
                                   grid[i].seg_bits};
        set_knobs(v);
        ActiveCtx active(ctx);
        rc = pd_sort_dev(ctx, in, nsets, p, part_begin, opts, &r, st);  // warm: scratch grows here
        double t = 1e300;
        for (uint32_t k = 0; k < trials && rc == DSSS_OK; ++k) {
            cudaEventRecord(e0, st);
            rc = pd_sort_dev(ctx, in, nsets, p, part_begin, opts, &r, st);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < t) t = ms;
        }
        if (rc != DSSS_OK) break;
        ++tried;
        if (i == 0) first = t;
        if (t < best) {
            best = t;
            best_i = i;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dev);
    if (rc != DSSS_OK || best_i < 0) {
        set_knobs(saved.v);
        return rc != DSSS_OK ? rc : fail(DSSS_EDEVICE, "autotune: no setting ran");
    }
    const int64_t v[NKNOBS] = {grid[best_i].small_max, grid[best_i].pivot, grid[best_i].split_min, grid[best_i].bits,
                               grid[best_i].seg_bits};
    set_knobs(v);
    out->sort_small_max = v[0];
    out->sort_pivot = v[1];
    out->sort_split_min = v[2];
    out->sort_bits = v[3];
    out->sort_seg_bits = v[4];
    dsss_tune_get("dp_filter_min", &out->dp_filter_min);
    out->best_ms = best;
    out->default_ms = first;
    out->settings_tried = tried;
    return DSSS_OK;
}
