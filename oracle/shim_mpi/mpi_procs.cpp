// Process-based MPI subset (see mpi.h for the model).  Test infrastructure
// and the timed CPU reference arm only.
#include "mpi.h"

#include <fcntl.h>
#include <linux/futex.h>
#include <signal.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/stat.h>
#include <sys/syscall.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

namespace {

constexpr int kMaxRanks = 1024;
constexpr uint32_t kDescPerRank = 1u << 14;
constexpr uint64_t kCollBit = 1ull << 63;

struct Desc {
    uint64_t ctx;
    uint64_t bytes;
    uint64_t off;  // payload offset in the sender's arena region
    int32_t src;   // sender's rank in the communicator
    int32_t tag;
    int32_t next;  // next descriptor in the receiver's mailbox, -1 at the end
    std::atomic<int32_t> state;  // 0 free, 1 queued
};

struct alignas(64) Mailbox {
    std::atomic<int32_t> lock;
    std::atomic<uint32_t> bell;     // bumped on every arrival and every consumed send
    std::atomic<int32_t> sleeping;  // the owner is (about to be) in futex_wait
    int32_t head, tail;
};

struct alignas(64) SenderState {
    std::atomic<int64_t> live;  // this rank's messages not yet consumed
};

struct Ctl {
    int32_t np;
    std::atomic<int32_t> abort_flag;
    int32_t pids[kMaxRanks];
    std::atomic<int32_t> finalized[kMaxRanks];  // set by a rank just before it exits
    Mailbox box[kMaxRanks];
    SenderState snd[kMaxRanks];
    // followed by np * kDescPerRank descriptors
};

Ctl* g_ctl = nullptr;
Desc* g_desc = nullptr;
unsigned char* g_arena = nullptr;
uint64_t g_arena_bytes = 0;  // per rank
int g_me = 0, g_np = 1;
bool g_init = false, g_final = false;
std::vector<char> g_reaped;  // rank 0: children already collected
uint64_t g_top = 0;          // bump pointer in my arena region
uint32_t g_desc_cursor = 0;
double g_timeout = 900.0;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] void fatal(const char* what) {
    std::fprintf(stderr, "[rank %d] MPI stand-in: %s\n", g_me, what);
    std::fflush(stderr);
    if (g_ctl) {
        g_ctl->abort_flag.store(1);
        for (int r = 0; r < g_np; ++r)
            if (r != g_me && g_ctl->pids[r] > 0) kill(g_ctl->pids[r], SIGKILL);
    }
    _exit(2);
}

void check_alive() {
    if (g_ctl->abort_flag.load(std::memory_order_relaxed)) _exit(2);
    if (g_me == 0) {
        int st = 0;
        pid_t p = waitpid(-1, &st, WNOHANG);
        if (p > 0) {
            int r = 1;
            while (r < g_np && g_ctl->pids[r] != p) ++r;
            if (r < g_np) {
                if (!(WIFEXITED(st) && WEXITSTATUS(st) == 0) || !g_ctl->finalized[r].load())
                    fatal("a rank ended before MPI_Finalize");
                g_reaped[r] = 1;
            }
        }
    } else if (getppid() != g_ctl->pids[0]) {
        _exit(2);
    }
}

long futex(std::atomic<uint32_t>* addr, int op, uint32_t val, const struct timespec* ts) {
    return syscall(SYS_futex, reinterpret_cast<uint32_t*>(addr), op, val, ts, nullptr, 0);
}

void ring(int world_rank) {
    Mailbox& b = g_ctl->box[world_rank];
    b.bell.fetch_add(1, std::memory_order_seq_cst);
    if (b.sleeping.load(std::memory_order_seq_cst)) futex(&b.bell, FUTEX_WAKE, 1 << 30, nullptr);
}

// Runs `ready` until it returns true, sleeping on this rank's bell between tries.
template <typename F>
void wait_until(F&& ready) {
    Mailbox& b = g_ctl->box[g_me];
    const double t0 = now_s();
    for (int spins = 0;; ++spins) {
        uint32_t seen = b.bell.load(std::memory_order_seq_cst);
        if (ready()) return;
        if (spins < 64) continue;
        check_alive();
        if (now_s() - t0 > g_timeout) fatal("timed out waiting for a message");
        b.sleeping.store(1, std::memory_order_seq_cst);
        if (ready()) {
            b.sleeping.store(0, std::memory_order_seq_cst);
            return;
        }
        struct timespec ts = {0, 20 * 1000 * 1000};
        futex(&b.bell, FUTEX_WAIT, seen, &ts);
        b.sleeping.store(0, std::memory_order_seq_cst);
    }
}

void lock(std::atomic<int32_t>& l) {
    for (int k = 0;; ++k) {
        int32_t z = 0;
        if (l.compare_exchange_weak(z, 1, std::memory_order_acquire)) return;
        if (k > 32) sched_yield();
    }
}
void unlock(std::atomic<int32_t>& l) { l.store(0, std::memory_order_release); }

// ---------------------------------------------------------------- datatypes
std::vector<int64_t> g_types;     // derived type sizes
std::vector<int32_t> g_type_free;
int64_t type_size(MPI_Datatype t) {
    if (t < 0x10000) return t & 0xff;
    size_t i = (size_t)(t - 0x10000);
    if (i >= g_types.size() || g_types[i] < 0) fatal("unknown datatype");
    return g_types[i];
}
MPI_Datatype new_type(int64_t size) {
    if (!g_type_free.empty()) {
        int32_t i = g_type_free.back();
        g_type_free.pop_back();
        g_types[i] = size;
        return 0x10000 + i;
    }
    g_types.push_back(size);
    return 0x10000 + (int)g_types.size() - 1;
}

// ---------------------------------------------------------------- communicators
struct Comm {
    uint64_t ctx;
    int rank, size;
    std::vector<int> world;  // world rank of each member
    uint32_t coll_seq = 0, split_seq = 0;
    bool used = false;
};
std::vector<Comm> g_comms;

uint64_t mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

Comm& comm_of(MPI_Comm c) {
    if (c <= 0 || (size_t)c >= g_comms.size() || !g_comms[c].used) fatal("invalid communicator");
    return g_comms[c];
}

// ---------------------------------------------------------------- messages
bool progress();
uint64_t arena_alloc(uint64_t bytes) {
    bytes = (bytes + 63) & ~63ull;
    if (bytes > g_arena_bytes) fatal("message larger than the arena (raise DSSS_MPI_ARENA_GB)");
    auto& live = g_ctl->snd[g_me].live;
    if (live.load(std::memory_order_acquire) == 0) g_top = 0;
    if (g_top + bytes > g_arena_bytes) {
        wait_until([&] { progress(); return live.load(std::memory_order_acquire) == 0; });
        g_top = 0;
    }
    uint64_t off = g_top;
    g_top += bytes;
    return off;
}

int32_t desc_alloc() {
    Desc* mine = g_desc + (size_t)g_me * kDescPerRank;
    int32_t found = -1;
    auto scan = [&] {
        for (uint32_t k = 0; k < kDescPerRank; ++k) {
            uint32_t i = (g_desc_cursor + k) % kDescPerRank;
            if (mine[i].state.load(std::memory_order_acquire) == 0) {
                g_desc_cursor = (i + 1) % kDescPerRank;
                found = (int32_t)((size_t)g_me * kDescPerRank + i);
                return true;
            }
        }
        return false;
    };
    if (!scan()) wait_until(scan);
    return found;
}

void post_send(const void* buf, uint64_t bytes, int dest_world, uint64_t ctx, int src_rank, int tag) {
    uint64_t off = arena_alloc(bytes);
    if (bytes) std::memcpy(g_arena + (size_t)g_me * g_arena_bytes + off, buf, bytes);
    int32_t d = desc_alloc();
    Desc& m = g_desc[d];
    m.ctx = ctx;
    m.bytes = bytes;
    m.off = off;
    m.src = src_rank;
    m.tag = tag;
    m.next = -1;
    m.state.store(1, std::memory_order_relaxed);
    g_ctl->snd[g_me].live.fetch_add(1, std::memory_order_acq_rel);
    Mailbox& b = g_ctl->box[dest_world];
    lock(b.lock);
    if (b.tail < 0) {
        b.head = b.tail = d;
    } else {
        g_desc[b.tail].next = d;
        b.tail = d;
    }
    unlock(b.lock);
    ring(dest_world);
}

// First message in my mailbox matching (ctx, src, tag); unlinked when `take`.
int32_t find_msg(uint64_t ctx, int src, int tag, bool take) {
    Mailbox& b = g_ctl->box[g_me];
    lock(b.lock);
    int32_t prev = -1, i = b.head;
    while (i >= 0) {
        const Desc& m = g_desc[i];
        if (m.ctx == ctx && (src == MPI_ANY_SOURCE || m.src == src) && (tag == MPI_ANY_TAG || m.tag == tag)) break;
        prev = i;
        i = m.next;
    }
    if (i >= 0 && take) {
        int32_t nx = g_desc[i].next;
        if (prev < 0) b.head = nx; else g_desc[prev].next = nx;
        if (b.tail == i) b.tail = prev;
    }
    unlock(b.lock);
    return i;
}

void consume(int32_t d, void* buf, uint64_t cap, MPI_Status* st) {
    Desc& m = g_desc[d];
    if (m.bytes > cap) fatal("message truncated: the receive buffer is smaller than the message");
    int sender = d / (int32_t)kDescPerRank;
    if (m.bytes) std::memcpy(buf, g_arena + (size_t)sender * g_arena_bytes + m.off, m.bytes);
    if (st) {
        st->MPI_SOURCE = m.src;
        st->MPI_TAG = m.tag;
        st->MPI_ERROR = 0;
        st->dsss_bytes = (long long)m.bytes;
    }
    m.state.store(0, std::memory_order_release);
    g_ctl->snd[sender].live.fetch_sub(1, std::memory_order_acq_rel);
    ring(sender);
}

// ---------------------------------------------------------------- requests
struct Req {
    int kind = 0;  // 0 free, 1 completed send, 2 receive
    void* buf = nullptr;
    uint64_t cap = 0;
    uint64_t ctx = 0;
    int src = 0, tag = 0;
    bool done = false;
    MPI_Status st{};
};
std::vector<Req> g_reqs(1);
std::vector<int> g_req_free;
std::vector<int> g_pending;  // posted receives in posting order

int req_new() {
    if (!g_req_free.empty()) {
        int i = g_req_free.back();
        g_req_free.pop_back();
        g_reqs[i] = Req();
        return i;
    }
    g_reqs.emplace_back();
    return (int)g_reqs.size() - 1;
}

// Serves posted receives in posting order; returns true if any completed.
bool progress() {
    bool any = false;
    for (size_t k = 0; k < g_pending.size();) {
        Req& r = g_reqs[g_pending[k]];
        int32_t d = find_msg(r.ctx, r.src, r.tag, true);
        if (d >= 0) {
            consume(d, r.buf, r.cap, &r.st);
            r.done = true;
            any = true;
            g_pending.erase(g_pending.begin() + (long)k);
        } else {
            ++k;
        }
    }
    return any;
}

int post_recv(void* buf, uint64_t cap, uint64_t ctx, int src, int tag) {
    int i = req_new();
    Req& r = g_reqs[i];
    r.kind = 2;
    r.buf = buf;
    r.cap = cap;
    r.ctx = ctx;
    r.src = src;
    r.tag = tag;
    g_pending.push_back(i);
    return i;
}

void finish_req(MPI_Request* h, MPI_Status* st) {
    int i = *h;
    if (i == MPI_REQUEST_NULL) return;
    Req& r = g_reqs[i];
    if (st) {
        if (r.kind == 2) *st = r.st;
        else { st->MPI_SOURCE = 0; st->MPI_TAG = 0; st->MPI_ERROR = 0; st->dsss_bytes = 0; }
    }
    r.kind = 0;
    g_req_free.push_back(i);
    *h = MPI_REQUEST_NULL;
}

void wait_req(int i) {
    if (g_reqs[i].kind != 2) return;
    progress();
    if (!g_reqs[i].done) wait_until([&] { progress(); return g_reqs[i].done; });
}

void recv_blocking(void* buf, uint64_t cap, uint64_t ctx, int src, int tag, MPI_Status* st) {
    int i = post_recv(buf, cap, ctx, src, tag);
    wait_req(i);
    MPI_Request h = i;
    finish_req(&h, st);
}

// ---------------------------------------------------------------- collectives
struct Coll {
    Comm& c;
    uint64_t ctx;
    int tag;
    explicit Coll(MPI_Comm comm) : c(comm_of(comm)) {
        ctx = c.ctx | kCollBit;
        tag = (int)(c.coll_seq++ & 0x3fffffff);
    }
    void send(int to, const void* buf, uint64_t bytes) { post_send(buf, bytes, c.world[to], ctx, c.rank, tag); }
    void recv(int from, void* buf, uint64_t cap) { recv_blocking(buf, cap, ctx, from, tag, nullptr); }
};

void alltoallv_bytes(MPI_Comm comm, const unsigned char* sb, const std::vector<uint64_t>& sc,
                     const std::vector<uint64_t>& sd, unsigned char* rb, const std::vector<uint64_t>& rc,
                     const std::vector<uint64_t>& rd) {
    Coll k(comm);
    const int P = k.c.size, me = k.c.rank;
    for (int j = 1; j < P; ++j) {
        int to = (me + j) % P;
        k.send(to, sb + sd[to], sc[to]);
    }
    if (sc[me] != rc[me]) fatal("alltoallv: own send and receive counts differ");
    if (sc[me]) std::memmove(rb + rd[me], sb + sd[me], sc[me]);
    for (int j = 1; j < P; ++j) {
        int from = (me - j + P) % P;
        k.recv(from, rb + rd[from], rc[from]);
    }
}

void allgather_bytes(MPI_Comm comm, const void* sb, uint64_t bytes, unsigned char* rb,
                     const std::vector<uint64_t>& rc, const std::vector<uint64_t>& rd) {
    Coll k(comm);
    const int P = k.c.size, me = k.c.rank;
    for (int j = 1; j < P; ++j) k.send((me + j) % P, sb, bytes);
    if (rc[me] != bytes) fatal("allgather: own count differs");
    if (bytes) std::memmove(rb + rd[me], sb, bytes);
    for (int j = 1; j < P; ++j) {
        int from = (me - j + P) % P;
        k.recv(from, rb + rd[from], rc[from]);
    }
}

template <typename T>
void reduce_into(T* acc, const T* x, int n, MPI_Op op) {
    for (int i = 0; i < n; ++i) {
        switch (op) {
        case MPI_SUM: acc[i] = (T)(acc[i] + x[i]); break;
        case MPI_PROD: acc[i] = (T)(acc[i] * x[i]); break;
        case MPI_MAX: acc[i] = std::max(acc[i], x[i]); break;
        case MPI_MIN: acc[i] = std::min(acc[i], x[i]); break;
        case MPI_LAND: acc[i] = (T)(acc[i] != 0 && x[i] != 0); break;
        case MPI_LOR: acc[i] = (T)(acc[i] != 0 || x[i] != 0); break;
        default: fatal("unsupported reduction");
        }
    }
}
template <typename T>
void reduce_int_bits(T* acc, const T* x, int n, MPI_Op op) {
    if (op == MPI_BAND) { for (int i = 0; i < n; ++i) acc[i] &= x[i]; return; }
    if (op == MPI_BOR) { for (int i = 0; i < n; ++i) acc[i] |= x[i]; return; }
    reduce_into(acc, x, n, op);
}

void reduce_typed(void* acc, const void* x, int n, MPI_Datatype t, MPI_Op op) {
    switch (t) {
    case MPI_BYTE: case MPI_UNSIGNED_CHAR: reduce_int_bits((uint8_t*)acc, (const uint8_t*)x, n, op); break;
    case MPI_CHAR: reduce_int_bits((int8_t*)acc, (const int8_t*)x, n, op); break;
    case MPI_SHORT: reduce_int_bits((int16_t*)acc, (const int16_t*)x, n, op); break;
    case MPI_UNSIGNED_SHORT: reduce_int_bits((uint16_t*)acc, (const uint16_t*)x, n, op); break;
    case MPI_INT: reduce_int_bits((int32_t*)acc, (const int32_t*)x, n, op); break;
    case MPI_UNSIGNED: reduce_int_bits((uint32_t*)acc, (const uint32_t*)x, n, op); break;
    case MPI_LONG_LONG_INT: case MPI_LONG: reduce_int_bits((int64_t*)acc, (const int64_t*)x, n, op); break;
    case MPI_UNSIGNED_LONG_LONG: case MPI_UNSIGNED_LONG:
        reduce_int_bits((uint64_t*)acc, (const uint64_t*)x, n, op);
        break;
    case MPI_DOUBLE: reduce_into((double*)acc, (const double*)x, n, op); break;
    case MPI_FLOAT: reduce_into((float*)acc, (const float*)x, n, op); break;
    default: fatal("reduction on a derived datatype");
    }
}

// every rank's contribution, in rank order
std::vector<unsigned char> gather_all(MPI_Comm comm, const void* sb, uint64_t bytes) {
    Comm& c = comm_of(comm);
    std::vector<unsigned char> all(bytes * (size_t)c.size);
    std::vector<uint64_t> rc(c.size, bytes), rd(c.size);
    for (int r = 0; r < c.size; ++r) rd[r] = bytes * (uint64_t)r;
    allgather_bytes(comm, sb, bytes, all.data(), rc, rd);
    return all;
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) {
    if (g_init) return MPI_SUCCESS;
    const char* e = std::getenv("DSSS_MPI_NP");
    g_np = e ? std::atoi(e) : 1;
    if (g_np < 1 || g_np > kMaxRanks) fatal("DSSS_MPI_NP out of range");
    e = std::getenv("DSSS_MPI_ARENA_GB");
    g_arena_bytes = (uint64_t)(e ? std::atof(e) : 16.0) * (1ull << 30);
    e = std::getenv("DSSS_MPI_TIMEOUT");
    if (e) g_timeout = std::atof(e);
    size_t ctl_bytes = sizeof(Ctl) + (size_t)g_np * kDescPerRank * sizeof(Desc);
    void* p = mmap(nullptr, ctl_bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (p == MAP_FAILED) fatal("mmap of the control block failed");
    g_ctl = static_cast<Ctl*>(p);
    g_desc = reinterpret_cast<Desc*>(static_cast<unsigned char*>(p) + sizeof(Ctl));
    g_ctl->np = g_np;
    for (int r = 0; r < g_np; ++r) {
        g_ctl->box[r].head = g_ctl->box[r].tail = -1;
    }
    int fd = (int)syscall(SYS_memfd_create, "dsss_mpi_arena", 0);
    if (fd < 0) fatal("memfd_create failed");
    if (ftruncate(fd, (off_t)(g_arena_bytes * (uint64_t)g_np)) != 0) fatal("ftruncate of the arena failed");
    void* a = mmap(nullptr, g_arena_bytes * (uint64_t)g_np, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_NORESERVE, fd, 0);
    if (a == MAP_FAILED) fatal("mmap of the arena failed");
    close(fd);
    g_arena = static_cast<unsigned char*>(a);
    g_ctl->pids[0] = getpid();
    g_reaped.assign(g_np, 0);
    std::cout.flush();
    std::cerr.flush();
    std::fflush(nullptr);
    for (int r = 1; r < g_np; ++r) {
        pid_t pid = fork();
        if (pid < 0) fatal("fork failed");
        if (pid == 0) {
            g_me = r;
            prctl(PR_SET_PDEATHSIG, SIGKILL);
            if (getppid() != g_ctl->pids[0]) _exit(2);
            break;
        }
        g_ctl->pids[r] = pid;
    }
    g_comms.resize(3);
    Comm& w = g_comms[MPI_COMM_WORLD];
    w.ctx = 2;
    w.rank = g_me;
    w.size = g_np;
    for (int r = 0; r < g_np; ++r) w.world.push_back(r);
    w.used = true;
    Comm& s = g_comms[MPI_COMM_SELF];
    s.ctx = mix(0x5E1Full + (uint64_t)g_me) & ~kCollBit;
    s.rank = 0;
    s.size = 1;
    s.world.push_back(g_me);
    s.used = true;
    g_init = true;
    // every rank's pid is published before anyone can time out
    MPI_Barrier(MPI_COMM_WORLD);
    return MPI_SUCCESS;
}

int MPI_Initialized(int* f) { *f = g_init ? 1 : 0; return MPI_SUCCESS; }
int MPI_Finalized(int* f) { *f = g_final ? 1 : 0; return MPI_SUCCESS; }

int MPI_Finalize(void) {
    if (!g_init || g_final) return MPI_SUCCESS;
    MPI_Barrier(MPI_COMM_WORLD);
    g_final = true;
    std::cout.flush();
    std::cerr.flush();
    std::fflush(nullptr);
    if (g_me != 0) {
        g_ctl->finalized[g_me].store(1);
        _exit(0);
    }
    bool bad = false;
    for (int r = 1; r < g_np; ++r) {
        if (g_reaped[r]) continue;
        int st = 0;
        if (waitpid(g_ctl->pids[r], &st, 0) != g_ctl->pids[r] || !WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = true;
    }
    if (bad) {
        std::fprintf(stderr, "MPI stand-in: a rank failed\n");
        _exit(2);
    }
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int) { fatal("MPI_Abort"); }

double MPI_Wtime(void) { return now_s(); }

int MPI_Comm_rank(MPI_Comm c, int* r) { *r = comm_of(c).rank; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int* s) { *s = comm_of(c).size; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out) {
    Comm& c = comm_of(comm);
    const uint32_t seq = c.split_seq++;
    int mine[2] = {color, key};
    std::vector<unsigned char> all = gather_all(comm, mine, sizeof(mine));
    const int* v = reinterpret_cast<const int*>(all.data());
    if (color == MPI_UNDEFINED) {
        *out = MPI_COMM_NULL;
        return MPI_SUCCESS;
    }
    std::vector<std::pair<std::pair<int, int>, int>> members;  // ((key, rank), rank)
    for (int r = 0; r < c.size; ++r)
        if (v[2 * r] == color) members.push_back({{v[2 * r + 1], r}, r});
    std::sort(members.begin(), members.end());
    Comm n;
    n.ctx = mix(mix(c.ctx ^ 0xC0117ull) + seq * 0x100000001ull + (uint64_t)(uint32_t)color) & ~kCollBit;
    if (n.ctx <= 2) n.ctx += 3;
    n.size = (int)members.size();
    for (int i = 0; i < n.size; ++i) {
        if (members[i].second == c.rank) n.rank = i;
        n.world.push_back(c.world[members[i].second]);
    }
    n.used = true;
    g_comms.push_back(n);
    *out = (int)g_comms.size() - 1;
    return MPI_SUCCESS;
}

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) {
    int r = 0;
    MPI_Comm_rank(comm, &r);
    return MPI_Comm_split(comm, 0, r, out);
}

int MPI_Comm_free(MPI_Comm* c) {
    if (*c > MPI_COMM_SELF && (size_t)*c < g_comms.size()) g_comms[*c].used = false;
    *c = MPI_COMM_NULL;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    Comm& c = comm_of(comm);
    std::vector<uint64_t> rc(c.size, 0), rd(c.size, 0);
    unsigned char dummy = 0;
    allgather_bytes(comm, &dummy, 0, &dummy, rc, rd);
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* nt) {
    *nt = new_type((int64_t)count * type_size(old));
    return MPI_SUCCESS;
}
int MPI_Type_create_struct(int count, const int* bl, const MPI_Aint* disp, const MPI_Datatype* ts, MPI_Datatype* nt) {
    int64_t ext = 0;
    for (int i = 0; i < count; ++i) ext = std::max<int64_t>(ext, disp[i] + (int64_t)bl[i] * type_size(ts[i]));
    *nt = new_type(ext);
    return MPI_SUCCESS;
}
int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint* lb, MPI_Aint* ext) {
    *lb = 0;
    *ext = type_size(t);
    return MPI_SUCCESS;
}
int MPI_Type_size(MPI_Datatype t, int* s) { *s = (int)type_size(t); return MPI_SUCCESS; }
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype* t) {
    if (*t >= 0x10000) {
        size_t i = (size_t)(*t - 0x10000);
        if (i < g_types.size() && g_types[i] >= 0) {
            g_types[i] = -1;
            g_type_free.push_back((int32_t)i);
        }
    }
    *t = 0;
    return MPI_SUCCESS;
}

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    if (dest < 0 || dest >= c.size) fatal("MPI_Send: bad destination");
    post_send(buf, (uint64_t)count * type_size(t), c.world[dest], c.ctx, c.rank, tag);
    return MPI_SUCCESS;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request* req) {
    MPI_Send(buf, count, t, dest, tag, comm);
    int i = req_new();
    g_reqs[i].kind = 1;
    g_reqs[i].done = true;
    *req = i;
    return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status* st) {
    Comm& c = comm_of(comm);
    recv_blocking(buf, (uint64_t)count * type_size(t), c.ctx, src, tag, st);
    return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Request* req) {
    Comm& c = comm_of(comm);
    *req = post_recv(buf, (uint64_t)count * type_size(t), c.ctx, src, tag);
    progress();
    return MPI_SUCCESS;
}
int MPI_Sendrecv(const void* sb, int sc, MPI_Datatype st_, int dest, int stag, void* rb, int rc, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm comm, MPI_Status* st) {
    MPI_Send(sb, sc, st_, dest, stag, comm);
    return MPI_Recv(rb, rc, rt, src, rtag, comm, st);
}
int MPI_Iprobe(int src, int tag, MPI_Comm comm, int* flag, MPI_Status* st) {
    Comm& c = comm_of(comm);
    progress();
    int32_t d = find_msg(c.ctx, src, tag, false);
    *flag = d >= 0;
    if (d >= 0 && st) {
        st->MPI_SOURCE = g_desc[d].src;
        st->MPI_TAG = g_desc[d].tag;
        st->MPI_ERROR = 0;
        st->dsss_bytes = (long long)g_desc[d].bytes;
    }
    return MPI_SUCCESS;
}
int MPI_Probe(int src, int tag, MPI_Comm comm, MPI_Status* st) {
    int flag = 0;
    MPI_Status tmp;
    wait_until([&] { MPI_Iprobe(src, tag, comm, &flag, &tmp); return flag != 0; });
    if (st) *st = tmp;
    return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* count) {
    int64_t s = type_size(t);
    *count = (s == 0 || st->dsss_bytes % s) ? MPI_UNDEFINED : (int)(st->dsss_bytes / s);
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status* st) {
    if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
    wait_req(*req);
    finish_req(req, st);
    return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* sts) {
    auto all_done = [&] {
        progress();
        for (int i = 0; i < count; ++i)
            if (reqs[i] != MPI_REQUEST_NULL && g_reqs[reqs[i]].kind == 2 && !g_reqs[reqs[i]].done) return false;
        return true;
    };
    if (!all_done()) wait_until(all_done);
    for (int i = 0; i < count; ++i) finish_req(&reqs[i], sts ? &sts[i] : nullptr);
    return MPI_SUCCESS;
}
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* st) {
    if (*req == MPI_REQUEST_NULL) { *flag = 1; return MPI_SUCCESS; }
    progress();
    Req& r = g_reqs[*req];
    *flag = (r.kind != 2 || r.done) ? 1 : 0;
    if (*flag) finish_req(req, st);
    return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
    Coll k(comm);
    uint64_t bytes = (uint64_t)count * type_size(t);
    if (k.c.rank == root) {
        for (int r = 0; r < k.c.size; ++r)
            if (r != root) k.send(r, buf, bytes);
    } else {
        k.recv(root, buf, bytes);
    }
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int* rcounts, const int* displs,
                MPI_Datatype rt, int root, MPI_Comm comm) {
    Coll k(comm);
    uint64_t sbytes = (uint64_t)sc * type_size(st);
    if (k.c.rank != root) {
        k.send(root, sb, sbytes);
        return MPI_SUCCESS;
    }
    int64_t es = type_size(rt);
    for (int r = 0; r < k.c.size; ++r) {
        unsigned char* dst = static_cast<unsigned char*>(rb) + (int64_t)displs[r] * es;
        if (r == root) {
            if (sbytes) std::memmove(dst, sb, sbytes);
        } else {
            k.recv(r, dst, (uint64_t)rcounts[r] * es);
        }
    }
    return MPI_SUCCESS;
}
int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, int root, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    std::vector<int> counts(c.size, rc), displs(c.size);
    for (int r = 0; r < c.size; ++r) displs[r] = r * rc;
    return MPI_Gatherv(sb, sc, st, rb, counts.data(), displs.data(), rt, root, comm);
}
int MPI_Scatter(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, int root, MPI_Comm comm) {
    Coll k(comm);
    uint64_t sbytes = (uint64_t)sc * type_size(st);
    if (k.c.rank == root) {
        for (int r = 0; r < k.c.size; ++r) {
            const unsigned char* src = static_cast<const unsigned char*>(sb) + sbytes * (uint64_t)r;
            if (r == root) {
                if (sbytes) std::memmove(rb, src, sbytes);
            } else {
                k.send(r, src, sbytes);
            }
        }
    } else {
        k.recv(root, rb, (uint64_t)rc * type_size(rt));
    }
    return MPI_SUCCESS;
}

int MPI_Allgatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int* rcounts, const int* displs,
                   MPI_Datatype rt, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    int64_t es = type_size(rt);
    std::vector<uint64_t> rc(c.size), rd(c.size);
    for (int r = 0; r < c.size; ++r) {
        rc[r] = (uint64_t)rcounts[r] * es;
        rd[r] = (uint64_t)((int64_t)displs[r] * es);
    }
    allgather_bytes(comm, sb, (uint64_t)sc * type_size(st), static_cast<unsigned char*>(rb), rc, rd);
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    int64_t es = type_size(rt);
    std::vector<uint64_t> cnt(c.size, (uint64_t)rc * es), dsp(c.size);
    for (int r = 0; r < c.size; ++r) dsp[r] = (uint64_t)rc * es * (uint64_t)r;
    allgather_bytes(comm, sb, (uint64_t)sc * type_size(st), static_cast<unsigned char*>(rb), cnt, dsp);
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void* sb, const int* scounts, const int* sdispls, MPI_Datatype st, void* rb,
                  const int* rcounts, const int* rdispls, MPI_Datatype rt, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    int64_t ss = type_size(st), rs = type_size(rt);
    std::vector<uint64_t> sc(c.size), sd(c.size), rc(c.size), rd(c.size);
    for (int r = 0; r < c.size; ++r) {
        sc[r] = (uint64_t)scounts[r] * ss;
        sd[r] = (uint64_t)((int64_t)sdispls[r] * ss);
        rc[r] = (uint64_t)rcounts[r] * rs;
        rd[r] = (uint64_t)((int64_t)rdispls[r] * rs);
    }
    alltoallv_bytes(comm, static_cast<const unsigned char*>(sb), sc, sd, static_cast<unsigned char*>(rb), rc, rd);
    return MPI_SUCCESS;
}
int MPI_Alltoall(const void* sb, int scount, MPI_Datatype st, void* rb, int rcount, MPI_Datatype rt, MPI_Comm comm) {
    Comm& c = comm_of(comm);
    int64_t ss = (int64_t)scount * type_size(st), rs = (int64_t)rcount * type_size(rt);
    std::vector<uint64_t> sc(c.size, ss), sd(c.size), rc(c.size, rs), rd(c.size);
    for (int r = 0; r < c.size; ++r) {
        sd[r] = (uint64_t)(ss * r);
        rd[r] = (uint64_t)(rs * r);
    }
    alltoallv_bytes(comm, static_cast<const unsigned char*>(sb), sc, sd, static_cast<unsigned char*>(rb), rc, rd);
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
    uint64_t bytes = (uint64_t)count * type_size(t);
    std::vector<unsigned char> all = gather_all(comm, sb, bytes);
    Comm& c = comm_of(comm);
    std::vector<unsigned char> acc(all.begin(), all.begin() + (long)bytes);
    for (int r = 1; r < c.size; ++r) reduce_typed(acc.data(), all.data() + bytes * (uint64_t)r, count, t, op);
    if (bytes) std::memcpy(rb, acc.data(), bytes);
    return MPI_SUCCESS;
}
int MPI_Reduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm) {
    uint64_t bytes = (uint64_t)count * type_size(t);
    std::vector<unsigned char> tmp(bytes);
    MPI_Allreduce(sb, tmp.data(), count, t, op, comm);
    if (comm_of(comm).rank == root && bytes) std::memcpy(rb, tmp.data(), bytes);
    return MPI_SUCCESS;
}
int MPI_Scan(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
    uint64_t bytes = (uint64_t)count * type_size(t);
    std::vector<unsigned char> all = gather_all(comm, sb, bytes);
    Comm& c = comm_of(comm);
    std::vector<unsigned char> acc(all.begin(), all.begin() + (long)bytes);
    for (int r = 1; r <= c.rank; ++r) reduce_typed(acc.data(), all.data() + bytes * (uint64_t)r, count, t, op);
    if (bytes) std::memcpy(rb, acc.data(), bytes);
    return MPI_SUCCESS;
}
int MPI_Exscan(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
    uint64_t bytes = (uint64_t)count * type_size(t);
    std::vector<unsigned char> all = gather_all(comm, sb, bytes);
    Comm& c = comm_of(comm);
    if (c.rank == 0) return MPI_SUCCESS;  // undefined on rank 0, as in MPI
    std::vector<unsigned char> acc(all.begin(), all.begin() + (long)bytes);
    for (int r = 1; r < c.rank; ++r) reduce_typed(acc.data(), all.data() + bytes * (uint64_t)r, count, t, op);
    if (bytes) std::memcpy(rb, acc.data(), bytes);
    return MPI_SUCCESS;
}

// ---------------------------------------------------------------- MPI-IO (byte view only)
struct FileH {
    int fd = -1;
    int64_t pos = 0;
};
static std::vector<FileH> g_files(1);

int MPI_File_open(MPI_Comm, const char* name, int amode, MPI_Info, MPI_File* fh) {
    int flags = (amode & MPI_MODE_RDWR) ? O_RDWR : (amode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(name, flags, 0644);
    if (fd < 0) return 1;
    g_files.push_back({fd, 0});
    *fh = (int)g_files.size() - 1;
    return MPI_SUCCESS;
}
int MPI_File_close(MPI_File* fh) {
    if (*fh > 0 && (size_t)*fh < g_files.size() && g_files[*fh].fd >= 0) {
        close(g_files[*fh].fd);
        g_files[*fh].fd = -1;
    }
    *fh = 0;
    return MPI_SUCCESS;
}
int MPI_File_get_size(MPI_File fh, MPI_Offset* size) {
    struct stat s;
    if (fstat(g_files.at(fh).fd, &s) != 0) return 1;
    *size = (MPI_Offset)s.st_size;
    return MPI_SUCCESS;
}
int MPI_File_seek(MPI_File fh, MPI_Offset off, int) {
    g_files.at(fh).pos = off;
    return MPI_SUCCESS;
}
int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype t, MPI_Status* st) {
    FileH& f = g_files.at(fh);
    uint64_t want = (uint64_t)count * type_size(t), got = 0;
    while (got < want) {
        ssize_t r = pread(f.fd, static_cast<char*>(buf) + got, want - got, f.pos + (int64_t)got);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        got += (uint64_t)r;
    }
    f.pos += (int64_t)got;
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = 0; st->MPI_ERROR = 0; st->dsss_bytes = (long long)got; }
    return MPI_SUCCESS;
}
int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status* st) {
    FileH& f = g_files.at(fh);
    uint64_t want = (uint64_t)count * type_size(t), put = 0;
    while (put < want) {
        ssize_t r = pwrite(f.fd, static_cast<const char*>(buf) + put, want - put, f.pos + (int64_t)put);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        put += (uint64_t)r;
    }
    f.pos += (int64_t)put;
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = 0; st->MPI_ERROR = 0; st->dsss_bytes = (long long)put; }
    return MPI_SUCCESS;
}

}  // extern "C"
