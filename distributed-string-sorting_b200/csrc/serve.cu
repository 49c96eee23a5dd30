// Request server: continuous batching of sort requests onto one GPU.
//
// Clients submit string sets (host arenas) at any time.  Worker threads, each
// with its own stream and pinned staging, take the requests waiting at the
// head of the queue, as many as fit the batch limits and the device-memory
// budget, and run them as one dsss_pd_sort_batched call; several workers keep
// batches in flight at once, so the copies of one overlap the kernels of
// another and small batches share the device.  A request joins the next batch
// that a worker forms after it arrives, i.e. as soon as a worker and memory are
// free; the queue is served in arrival order (a request that does not fit
// waits and blocks the ones behind it, so none starves).
//
// Device memory comes from a CUDA memory pool whose release threshold is the
// budget: buffers freed after a batch stay resident for the next one.  The
// server admits a batch only if its whole footprint (input arena, outputs and
// pipeline scratch, computed exactly from the pipeline's layout) fits in the
// budget beside the batches in flight; a request that alone exceeds the budget
// completes with DSSS_ENOMEM.  Every request's result is the one a call of
// dsss_pd_sort_host on that request alone returns.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.cuh"
#include "pd.cuh"
#include "util.cuh"

namespace dsss {

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t id = 0;
    dsss_arena in{};
    std::vector<uint64_t> pb;  // p + 1 request-local PE bounds
    dsss_pd_result out{};
    dsss_request_stats st{};
    bool done = false;
};

// Set of every batched string (binary search over the nsets + 1 set bounds).
__device__ __forceinline__ uint32_t batch_set_of(const uint64_t* sb, uint32_t nsets, uint64_t i) {
    uint32_t lo = 0, hi = nsets;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sb[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Request-local char offsets -> offsets into the batch's char buffer.
__global__ void k_rebase_offsets(uint64_t* off, uint64_t n, const uint64_t* sb, const uint64_t* cbase,
                                 uint32_t nsets) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) off[i] += cbase[batch_set_of(sb, nsets, i)];
}

// Batch string ids -> request-local ids.
__global__ void k_local_ids(uint32_t* ids, uint64_t n, const uint64_t* sb, uint32_t nsets) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ids[i] -= (uint32_t)sb[batch_set_of(sb, nsets, i)];
}

// Device buffers of one batch ahead of the pipeline's scratch.
struct IoLayout {
    uint8_t* chars;
    uint64_t* off;
    uint32_t *len, *lorder, *dp, *pidx, *ppe, *mlcp;
    uint64_t *sb, *cb;
};

static uint64_t carve_io(Carve& c, IoLayout& L, uint64_t n, uint64_t chars, uint32_t nsets) {
    const uint64_t N = n ? n : 1;
    L.chars = c.take<uint8_t>(chars + 64);
    L.off = c.take<uint64_t>(N);
    L.len = c.take<uint32_t>(N);
    L.lorder = c.take<uint32_t>(N);
    L.dp = c.take<uint32_t>(N);
    L.pidx = c.take<uint32_t>(N);
    L.ppe = c.take<uint32_t>(N);
    L.mlcp = c.take<uint32_t>(N);
    L.sb = c.take<uint64_t>(nsets + 1);
    L.cb = c.take<uint64_t>(nsets + 1);
    return (c.used + 255) & ~255ull;
}

struct Batch {
    std::vector<Request*> reqs;
    uint64_t n = 0, chars = 0, footprint = 0;
};

struct Server {
    dsss_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1, next_batch = 1;
    uint64_t reserved = 0, max_reserved = 0;
    uint64_t batches = 0, batched_sets = 0;
    bool stop = false;
    cudaMemPool_t pool = nullptr;
    std::vector<std::thread> workers;

    // Device bytes a batch of the given requests holds while it runs: its
    // arena, outputs and the pipeline's scratch.
    uint64_t footprint(uint64_t n, uint64_t chars, uint32_t nsets) const {
        Carve c(nullptr);
        IoLayout L;
        return carve_io(c, L, n, chars, nsets) + pd_scratch_bytes(n, nsets, cfg.p, &cfg.opts);
    }
};

static uint64_t req_chars(const Request* r) { return (r->in.char_bytes + 255) & ~255ull; }

// Takes the requests at the head of the queue that fit one batch (mu held).
// Returns false if the head request cannot run yet (memory in use).
static bool form_batch(Server* s, Batch& b) {
    const uint32_t p = s->cfg.p;
    const uint32_t max_sets = std::min<uint32_t>(s->cfg.max_sets, MAX_SPLIT_BUCKETS / p);
    while (!s->queue.empty() && b.reqs.size() < max_sets) {
        Request* r = s->queue.front();
        const uint64_t n = b.n + r->in.n, chars = b.chars + req_chars(r);
        if (!b.reqs.empty() && s->cfg.max_batch_strings && n > s->cfg.max_batch_strings) break;
        const uint64_t f = s->footprint(n, chars, (uint32_t)b.reqs.size() + 1);
        if (s->reserved + f > s->cfg.hbm_budget) {
            if (b.reqs.empty() && s->footprint(r->in.n, req_chars(r), 1) > s->cfg.hbm_budget) {
                // can never run: fail it now
                s->queue.pop_front();
                r->st.status = DSSS_ENOMEM;
                snprintf(r->st.error, sizeof r->st.error, "request needs %llu device bytes, budget %llu",
                         (unsigned long long)s->footprint(r->in.n, req_chars(r), 1),
                         (unsigned long long)s->cfg.hbm_budget);
                r->st.t_done = now_s();
                r->done = true;
                s->cv_done.notify_all();
                continue;
            }
            break;
        }
        s->queue.pop_front();
        b.reqs.push_back(r);
        b.n = n;
        b.chars = chars;
        b.footprint = f;
    }
    return !b.reqs.empty();
}

// Runs one batch on the worker's stream; returns a status for all its requests.
static int run_batch(Server* s, Ctx* ctx, cudaStream_t st, Batch& b, uint64_t batch_id, double* t_copied,
                     double* t_sorted) {
    const uint32_t p = s->cfg.p, nsets = (uint32_t)b.reqs.size();
    const uint64_t n = b.n;
    void* block = nullptr;
    DSSS_CUDA(cudaMallocFromPoolAsync(&block, b.footprint, s->pool, st));
    struct Free {
        void* p;
        cudaStream_t st;
        ~Free() {
            if (p) cudaFreeAsync(p, st);
        }
    } guard{block, st};
    Carve c(block);
    IoLayout L;
    const uint64_t io = carve_io(c, L, n, b.chars, nsets);
    if (io > b.footprint) return fail(DSSS_EDEVICE, "server: batch layout exceeds its footprint");
    uint8_t* chars = L.chars;
    uint64_t *off = L.off, *sb_d = L.sb, *cb_d = L.cb;
    uint32_t *len = L.len, *lorder = L.lorder, *dp = L.dp, *pidx = L.pidx, *ppe = L.ppe, *mlcp = L.mlcp;

    std::vector<uint64_t> sb(nsets + 1, 0), cb(nsets + 1, 0), pb((uint64_t)nsets * p + 1, 0);
    for (uint32_t k = 0; k < nsets; ++k) {
        const Request* r = b.reqs[k];
        sb[k + 1] = sb[k] + r->in.n;
        cb[k + 1] = cb[k] + req_chars(r);
        for (uint32_t q = 0; q < p; ++q) pb[(uint64_t)k * p + q + 1] = sb[k] + r->pb[q + 1];
    }
    for (uint32_t k = 0; k < nsets; ++k) {
        const Request* r = b.reqs[k];
        if (r->in.char_bytes)
            DSSS_CUDA(cudaMemcpyAsync(chars + cb[k], r->in.chars, r->in.char_bytes, cudaMemcpyHostToDevice, st));
        if (r->in.n) {
            DSSS_CUDA(cudaMemcpyAsync(off + sb[k], r->in.offsets, r->in.n * 8, cudaMemcpyHostToDevice, st));
            DSSS_CUDA(cudaMemcpyAsync(len + sb[k], r->in.lengths, r->in.n * 4, cudaMemcpyHostToDevice, st));
        }
        // zero the gap up to the next set's 256-byte boundary (readable padding)
        const uint64_t end = cb[k] + r->in.char_bytes;
        DSSS_CUDA(cudaMemsetAsync(chars + end, 0, cb[k + 1] - end, st));
    }
    DSSS_CUDA(cudaMemsetAsync(chars + b.chars, 0, 64, st));
    DSSS_CUDA(cudaMemcpyAsync(sb_d, sb.data(), (nsets + 1) * 8, cudaMemcpyHostToDevice, st));
    DSSS_CUDA(cudaMemcpyAsync(cb_d, cb.data(), (nsets + 1) * 8, cudaMemcpyHostToDevice, st));
    if (n) DSSS_LAUNCH("k_rebase_offsets", st, k_rebase_offsets<<<grid_for(n, 256), 256, 0, st>>>(off, n, sb_d, cb_d, nsets));
    if (s->cfg.flags & DSSS_SERVER_TIMESTAMPS) {
        DSSS_CUDA(cudaStreamSynchronize(st));
        *t_copied = now_s();
    }

    dsss_arena a{chars, b.chars, off, len, n};
    std::vector<uint64_t> intervals((uint64_t)nsets * p * p), recv((uint64_t)nsets * p);
    dsss_pd_result dr{lorder, nullptr, dp, intervals.data(), pidx, ppe, mlcp, recv.data()};
    Ctx sub = *ctx;
    sub.ws = (char*)block + io;
    sub.ws_cap = b.footprint - io;
    sub.fixed_ws = true;
    int rc = pd_sort_dev(&sub, &a, nsets, p, pb.data(), &s->cfg.opts, &dr, st);
    ctx->pin = sub.pin;
    ctx->pin_cap = sub.pin_cap;
    if (rc != DSSS_OK) return rc;
    *t_sorted = now_s();  // pd_sort_dev returns after its last read-back
    if (n) DSSS_LAUNCH("k_local_ids", st, k_local_ids<<<grid_for(n, 256), 256, 0, st>>>(lorder, n, sb_d, nsets));
    for (uint32_t k = 0; k < nsets; ++k) {
        Request* r = b.reqs[k];
        const uint64_t m = r->in.n, o = sb[k];
        if (m) {
            DSSS_CUDA(cudaMemcpyAsync(r->out.local_order, lorder + o, m * 4, cudaMemcpyDeviceToHost, st));
            if (p > 1) {
                DSSS_CUDA(cudaMemcpyAsync(r->out.dp, dp + o, m * 4, cudaMemcpyDeviceToHost, st));
                DSSS_CUDA(cudaMemcpyAsync(r->out.perm_index, pidx + o, m * 4, cudaMemcpyDeviceToHost, st));
                DSSS_CUDA(cudaMemcpyAsync(r->out.perm_pe, ppe + o, m * 4, cudaMemcpyDeviceToHost, st));
                if (r->out.merged_lcp)
                    DSSS_CUDA(cudaMemcpyAsync(r->out.merged_lcp, mlcp + o, m * 4, cudaMemcpyDeviceToHost, st));
            }
        }
        if (p > 1 && r->out.intervals)
            std::memcpy(r->out.intervals, intervals.data() + (uint64_t)k * p * p, (uint64_t)p * p * 8);
        std::memcpy(r->out.recv_counts, recv.data() + (uint64_t)k * p, (uint64_t)p * 8);
    }
    DSSS_CUDA(cudaGetLastError());
    guard.p = nullptr;
    DSSS_CUDA(cudaFreeAsync(block, st));
    DSSS_CUDA(cudaStreamSynchronize(st));
    (void)batch_id;
    return DSSS_OK;
}

static void worker_main(Server* s) {
    Ctx ctx;
    ctx.device = s->cfg.device;
    cudaSetDevice(s->cfg.device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (;;) {
        Batch b;
        uint64_t batch_id = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop && s->queue.empty()) goto out;
                if (!s->queue.empty() && form_batch(s, b)) break;
                s->cv_work.wait(lk);
            }
            batch_id = s->next_batch++;
            s->reserved += b.footprint;
            s->max_reserved = std::max(s->max_reserved, s->reserved);
            s->batches += 1;
            s->batched_sets += b.reqs.size();
            const double t = now_s();
            for (Request* r : b.reqs) r->st.t_admit = t;
        }
        int rc;
        double t_copied = 0, t_sorted = 0;
        {
            ActiveCtx active(&ctx);
            rc = run_batch(s, &ctx, st, b, batch_id, &t_copied, &t_sorted);
        }
        char msg[sizeof(dsss_request_stats::error)] = "";
        if (rc != DSSS_OK) {
            snprintf(msg, sizeof msg, "%s", dsss_last_error());
            cudaStreamSynchronize(st);  // the batch's block may still be in use
            cudaGetLastError();
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->reserved -= b.footprint;
            const double t = now_s();
            for (Request* r : b.reqs) {
                r->st.status = rc;
                r->st.batch_id = batch_id;
                r->st.batch_sets = (uint32_t)b.reqs.size();
                r->st.batch_strings = b.n;
                r->st.t_done = t;
                r->st.t_copied = t_copied;
                r->st.t_sorted = t_sorted;
                if (rc != DSSS_OK) snprintf(r->st.error, sizeof r->st.error, "%s", msg);
                r->done = true;
            }
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // memory came free: another worker may form a batch
    }
out:
    if (ctx.pin) cudaFreeHost(ctx.pin);
    if (st) cudaStreamDestroy(st);
}

}  // namespace dsss

using namespace dsss;

struct dsss_server {
    Server s;
};

extern "C" {

double dsss_clock_now(void) { return now_s(); }

int dsss_server_create(const dsss_server_config* cfg, dsss_server** out) {
    if (!cfg || !out) return fail(DSSS_EINVAL, "cfg/out is NULL");
    if (cfg->p == 0 || cfg->p > MAX_SPLIT_BUCKETS) return fail(DSSS_EINVAL, "p must be in 1..%u", MAX_SPLIT_BUCKETS);
    std::unique_ptr<dsss_server> h(new dsss_server);
    Server& s = h->s;
    s.cfg = *cfg;
    if (!s.cfg.workers) s.cfg.workers = 2;
    if (!s.cfg.max_sets) s.cfg.max_sets = MAX_SPLIT_BUCKETS / s.cfg.p;
    if (!s.cfg.hbm_budget) s.cfg.hbm_budget = 150000000000ull;
    DSSS_CUDA(cudaSetDevice(s.cfg.device));
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s.cfg.device;
    DSSS_CUDA(cudaMemPoolCreate(&s.pool, &props));
    uint64_t keep = s.cfg.hbm_budget;  // freed blocks stay resident up to the budget
    DSSS_CUDA(cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    if (s.cfg.reserve_bytes) {
        // map the reserve now: growing the pool later stalls the batches in flight
        const uint64_t r = std::min(s.cfg.reserve_bytes, s.cfg.hbm_budget);
        void* p = nullptr;
        cudaStream_t st = nullptr;
        DSSS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        cudaError_t e = cudaMallocFromPoolAsync(&p, r, s.pool, st);
        if (e == cudaSuccess) e = cudaFreeAsync(p, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaMemPoolDestroy(s.pool);
            return fail(DSSS_ENOMEM, "server: reserving %llu device bytes failed: %s", (unsigned long long)r,
                        cudaGetErrorString(e));
        }
    }
    for (uint32_t w = 0; w < s.cfg.workers; ++w) s.workers.emplace_back(worker_main, &s);
    *out = h.release();
    return DSSS_OK;
}

int dsss_server_submit(dsss_server* h, const dsss_arena* in, const uint64_t* part_begin, dsss_pd_result* out,
                       uint64_t* ticket) {
    if (!h || !ticket) return fail(DSSS_EINVAL, "server/ticket is NULL");
    Server& s = h->s;
    DSSS_TRY(check_arena(in));
    if (!out || !out->recv_counts || (in->n && !out->local_order))
        return fail(DSSS_EINVAL, "result arrays missing");
    if (s.cfg.p > 1 && in->n && (!out->dp || !out->perm_index || !out->perm_pe || !out->intervals))
        return fail(DSSS_EINVAL, "result arrays missing");
    const uint32_t p = s.cfg.p;
    std::unique_ptr<Request> r(new Request);
    r->in = *in;
    r->out = *out;
    r->pb.resize(p + 1);
    for (uint32_t q = 0; q <= p; ++q) r->pb[q] = part_begin ? part_begin[q] : (uint64_t)q * in->n / p;
    if (r->pb[0] != 0 || r->pb[p] != in->n) return fail(DSSS_EINVAL, "part_begin must start at 0 and end at n");
    for (uint32_t q = 0; q < p; ++q)
        if (r->pb[q + 1] < r->pb[q]) return fail(DSSS_EINVAL, "part_begin must be non-decreasing");
    r->st.status = 1;
    r->st.t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s.mu);
        if (s.stop) return fail(DSSS_EINVAL, "server is shutting down");
        r->id = s.next_id++;
        *ticket = r->id;
        s.queue.push_back(r.get());
        s.reqs.emplace(r->id, std::move(r));
    }
    s.cv_work.notify_one();
    return DSSS_OK;
}

int dsss_server_wait(dsss_server* h, uint64_t ticket, int64_t timeout_ms, dsss_request_stats* stats) {
    if (!h) return fail(DSSS_EINVAL, "server is NULL");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.reqs.find(ticket);
    if (it == s.reqs.end()) return fail(DSSS_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
    Request* r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) s.cv_done.wait(lk, ready);
    else if (!s.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return fail(DSSS_ETIMEDOUT, "request %llu not done after %lld ms", (unsigned long long)ticket,
                    (long long)timeout_ms);
    if (stats) *stats = r->st;
    const int rc = r->st.status;
    s.reqs.erase(it);
    if (rc != DSSS_OK) return fail(rc, "%s", stats ? stats->error : "request failed");
    return DSSS_OK;
}

int dsss_server_info(dsss_server* h, dsss_server_info_t* info) {
    if (!h || !info) return fail(DSSS_EINVAL, "server/info is NULL");
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    info->queued = s.queue.size();
    info->reserved_bytes = s.reserved;
    info->max_reserved_bytes = s.max_reserved;
    info->batches = s.batches;
    info->batched_requests = s.batched_sets;
    info->hbm_budget = s.cfg.hbm_budget;
    return DSSS_OK;
}

uint64_t dsss_server_footprint(dsss_server* h, uint64_t n, uint64_t char_bytes) {
    if (!h) return 0;
    return h->s.footprint(n, (char_bytes + 255) & ~255ull, 1);
}

int dsss_server_destroy(dsss_server* h) {
    if (!h) return DSSS_OK;
    Server& s = h->s;
    {
        std::lock_guard<std::mutex> lk(s.mu);
        s.stop = true;
    }
    s.cv_work.notify_all();
    for (auto& t : s.workers) t.join();
    if (s.pool) cudaMemPoolDestroy(s.pool);
    delete h;
    return DSSS_OK;
}

}  // extern "C"
