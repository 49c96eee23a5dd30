/*
 * dsss.h — C ABI of the B200 prefix-doubling string sorter.
 *
 * The reference (bingmann/distributed-string-sorting) exposes its hot path as
 * compile-time C++ policies; each entry point below replaces one of those
 * seams and cites the reference interface it stands in for.  One GPU holds
 * all p "PEs" (processing elements, the reference's MPI ranks) as contiguous
 * partitions of one string arena; the reference's all-to-all exchanges become
 * on-device scatters.
 *
 * Conventions
 *  - Strings live in an arena: bytes `chars`, per-string `offsets` (u64) and
 *    `lengths` (u32).  A string is chars[offsets[i] .. offsets[i]+lengths[i]);
 *    it must not contain byte 0 (the reference's strings are NUL-terminated,
 *    stringset.hpp:674-840).  Strings may overlap (suffix arrays).  Device
 *    arenas must be 8-byte aligned and readable 32 bytes past the last string
 *    byte (kernels use aligned vector loads); the *_host entry points pad for
 *    the caller.
 *  - PEs are contiguous index ranges: PE q owns strings [part_begin[q],
 *    part_begin[q+1]) (host array of p+1 entries, part_begin[0] = 0,
 *    part_begin[p] = n), like the reference's per-rank input slices.
 *  - n < 2^32 strings per call.  Index outputs are u32.
 *  - Return value: DSSS_OK (0) or a negative error code; dsss_last_error()
 *    gives a message for the calling thread.  The reference aborts instead
 *    (e.g. bloomfilter.hpp:595-600, merging.hpp:119-120).
 *  - Device entry points take device pointers and run on `stream`; they
 *    return after enqueuing, except where a size is needed on the host (the
 *    DP round loop and the partition step read small counts back).
 *  - A context owns reusable device scratch; use one context per host thread.
 */
#ifndef DSSS_H
#define DSSS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSSS_ABI_VERSION 1

#define DSSS_OK 0
#define DSSS_EINVAL (-22)
#define DSSS_ENOMEM (-12)
#define DSSS_ETIMEDOUT (-110)
#define DSSS_EDEVICE (-5)
#define DSSS_ENOTSUP (-95)

/* cudaStream_t without including CUDA headers (same underlying type). */
typedef struct CUstream_st* dsss_stream_t;

typedef struct dsss_ctx dsss_ctx;

typedef struct dsss_arena {
    const uint8_t* chars;    /* string bytes */
    uint64_t char_bytes;     /* bytes in chars that strings may reference */
    const uint64_t* offsets; /* [n] */
    const uint32_t* lengths; /* [n] */
    uint64_t n;
} dsss_arena;

/* Sampling policy of computePartition (samplingStrategies.hpp). */
#define DSSS_SAMPLER_NUM_STRINGS 0         /* SampleSplittersNumStringsPolicy :19-90 */
#define DSSS_SAMPLER_INDEXED_NUM_STRINGS 2 /* SampleIndexedSplittersNumStringsPolicy :106-186 */

typedef struct dsss_opts {
    uint32_t sampler;         /* DSSS_SAMPLER_* (prefix_doubling.cpp:359, default 0) */
    uint32_t sampling_factor; /* splitters per PE = factor*(p-1); the PD path uses 2 (prefix_doubling.hpp:251) */
    uint32_t small_sort_max;  /* string-sort knob: segments up to this size finish in one CTA (0 = default) */
    uint32_t flags;           /* DSSS_FLAG_* */
} dsss_opts;

#define DSSS_FLAG_LOCAL_LCP 1u /* dsss_pd_sort also writes local_lcp (costs one compare pass) */

/* Outputs of the full path, all device arrays of n entries unless noted.
 * NULL optional outputs are skipped. */
typedef struct dsss_pd_result {
    uint32_t* local_order;   /* per PE, the input index of each locally sorted string */
    uint32_t* local_lcp;     /* optional: LCP in local order, 0 at each PE start */
    uint32_t* dp;            /* distinguishing-prefix length per string, local order */
    uint64_t* intervals;     /* HOST [p*p]: strings PE q sends to PE r at [q*p + r] */
    uint32_t* perm_index;    /* merged output of PE 0, PE 1, ...: index into sender's local order */
    uint32_t* perm_pe;       /* ... and the sender PE */
    uint32_t* merged_lcp;    /* optional: LCP of merged neighbours, 0 at each PE start */
    uint64_t* recv_counts;   /* HOST [p]: merged strings per PE */
} dsss_pd_result;

/* ---- context ---------------------------------------------------------- */

/* hbm_budget_bytes: cap on scratch the context may hold (0 = no cap). */
int dsss_ctx_create(int device, uint64_t hbm_budget_bytes, dsss_ctx** out);
int dsss_ctx_destroy(dsss_ctx* ctx);
/* Scratch bytes currently held by the context. */
uint64_t dsss_ctx_scratch_bytes(const dsss_ctx* ctx);
const char* dsss_last_error(void);
/* Per-kernel timing (CUDA events around every launch of the calls made with
 * this context, on the launching stream).  on != 0 clears the totals. */
int dsss_ctx_set_timing(dsss_ctx* ctx, int on);
/* Lines "kernel launches total_ms" for the launches timed so far. */
int dsss_ctx_kernel_times(dsss_ctx* ctx, char* buf, uint64_t len);
int dsss_abi_version(void);

/* Process-wide tuning knobs (no reference counterpart), read by every later
 * call; value -1 restores the default.  Results never depend on them.
 *   dp_filter_min   hashed strings in a distinguishing-prefix round from which
 *                   duplicates are found through the fingerprint filter
 *                   (default 2^40, i.e. off: on B200 the filter's L2
 *                   atomics cost as much as the table's; 0 = always)
 *   dp_filter_bits  filter bits per hashed string (default 16)
 *   sort_small_max  small-segment cutoff of the string sort when dsss_opts
 *                   gives 0 (2..4096, default 4096)
 *   sort_pivot      pivot passes of the string sort on/off (default 1)
 *   dp_table        hash-table slots per hashed string in a distinguishing-
 *                   prefix round, rounded up to a power of two (2..8, default 2)
 *   sort_graph_max_n  largest n whose string sort runs as one CUDA graph with
 *                   a device-side pass loop (default 0 = never: measured on
 *                   B200 no faster than the host-driven loop, whose per-pass
 *                   read-back costs less than the graph's capacity-sized grids
 *                   and per-call instantiation)
 *   merge_by_sort   dsss_lcp_merge: decompressed runs merged by one segmented
 *                   string sort (1, default), by pairwise merge-path rounds
 *                   (0), or all p runs at once by co-ranked tiles (2: every
 *                   32nd string of every run sampled, the samples sorted, every
 *                   32nd sorted sample ranked in each run by binary search,
 *                   each tile of the runs' strings between two such bounds
 *                   sorted on its own from the bounds' common prefix);
 *                   identical results, ties in run order in every mode
 *   merge_extend_lanes  dsss_lcp_merge prefix decompression: threads that
 *                   decompress a chunk of 128 consecutive strings in order
 *                   (4, 8, 16 or 32; default 0 = from the average
 *                   decompressed length)
 *   dp_split        distinguishing-prefix hash rounds as two kernels, hashes
 *                   stored per position then inserted into the table (1), or
 *                   hash and insert in one kernel (0, default)
 *   copy_word       dsss_ms_sort / dsss_hq_sort: bytes per aligned store when
 *                   the output strings are copied out (16, default, or 8)
 *   dp_digest       distinguishing-prefix hash rounds in which at least 1/k
 *                   of the positions hash run in arena order: the hashed
 *                   strings are marked in a bitmap, hashed and inserted into
 *                   the table front to back (prefixes read in address order),
 *                   and the outcome read back as one bit per sorted position
 *                   (k = 1..64, default 4); 0 hashes every round by gathering
 *                   the prefixes in sorted order
 *   sort_split_min  smallest segment of the string sort's MSD passes that
 *                   may split by up to 255 splitters sampled from its keys
 *                   instead of by one key byte, where that byte takes few
 *                   values (letters, DNA; default 0 = never: on B200 the
 *                   fewer passes cost more in the small-segment sorts, whose
 *                   buckets then cut across key bytes; values below 4096
 *                   count as 4096)
 *   dp_check        1: the arena-order rounds at depths 8, 24, 40 and 72,
 *                   which read the prefix hashes the string sort's first pass
 *                   stored, recompute each from the string and fail with
 *                   DSSS_EDEVICE on a mismatch (a self-check; default 0)
 *   sort_bits       1: MSD passes over plain keys split on the eight most
 *                   significant bits in which a segment's keys differ (over
 *                   small alphabets one pass then covers more than a key
 *                   byte); 2: only where the first differing key byte varies
 *                   in at most four bits; 3: the same in the first pass only;
 *                   0: on the first differing key byte (default)
 *   sort_seg_bits   the same for the shared-memory passes of the segment
 *                   sorter (segments up to the small-segment cutoff; 0:
 *                   one key byte, the default) */
int dsss_tune_set(const char* name, int64_t value);
int dsss_tune_get(const char* name, int64_t* value);

/* Autotuner (no reference counterpart): runs the full path (as
 * dsss_pd_sort_batched; nsets = 1 for one set) on the given device input
 * under each setting of a grid of the knobs above (sort_small_max 256 / 1024 /
 * 4096, sort_pivot on / off, and the MSD digit: one key byte, sampled
 * splitters where a key byte splits poorly (sort_split_min 65536), the keys'
 * top differing bits in the passes over the arena where a byte varies in at
 * most four bits (sort_bits 2), in the first pass and inside the segment
 * sorter (sort_bits 3, sort_seg_bits 1), or inside the segment sorter only
 * (sort_seg_bits 1)),
 * 1 + trials runs each, and leaves the fastest setting in force for later
 * calls.  out: the chosen setting (dp_filter_min: the value in force, not
 * searched), its time (minimum over trials) and the default setting's
 * time. */
typedef struct {
    int64_t sort_small_max, sort_pivot, dp_filter_min;
    double best_ms, default_ms;
    uint32_t settings_tried;
    int64_t sort_split_min, sort_bits, sort_seg_bits;
} dsss_tuning;
int dsss_autotune(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p, const uint64_t* part_begin,
                  const dsss_opts* opts, uint32_t trials, dsss_tuning* out, dsss_stream_t stream);

/* ---- full path ---------------------------------------------------------- */

/* DistributedPrefixDoublingSort<...>::sort (src/sorter/distributed/prefix_doubling.hpp:200-295):
 * local sort, distinguishing prefixes, partition, exchange, merge, and the
 * (stringIndex, PEIndex) permutation (:282-290).  As in the reference, p == 1
 * stops after the local sort (:236): recv_counts[0] = 0, dp/perm untouched.
 * Byte-identical strings merge in (sender PE, local index) order; the
 * reference's loser tree orders them by tournament history instead. */
int dsss_pd_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                 const dsss_opts* opts, dsss_pd_result* out, dsss_stream_t stream);

/* Same with every array in host memory; copies in and out inside the call. */
int dsss_pd_sort_host(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                      const dsss_opts* opts, dsss_pd_result* out, dsss_stream_t stream);

/* Outputs of the merge-sort path, device arrays of n entries unless noted.
 * Receiving PEs back to back: PE r's recv_counts[r] strings, whole, in sorted
 * order. */
typedef struct dsss_ms_result {
    uint32_t* local_order;    /* per PE, the input index of each locally sorted string */
    uint64_t* intervals;      /* HOST [p*p]: strings PE q sends to PE r at [q*p + r] */
    uint8_t* chars;           /* the output strings, each followed by a NUL */
    uint64_t chars_capacity;  /* bytes at chars: at least the sum of (length + 1) */
    uint64_t* offsets;        /* start of each output string in chars */
    uint32_t* lengths;        /* length of each output string */
    uint32_t* lcp;            /* LCP with the previous output string, 0 at each PE start */
    uint32_t* source;         /* optional: input index of each output string */
    uint64_t* recv_counts;    /* HOST [p]: strings per receiving PE */
    uint64_t avg_lcp;         /* set by the call: getAvgLcp over all PEs */
} dsss_ms_result;

/* DistributedMergeSort<...>::sort (src/sorter/distributed/lcp_aware_number_string_splitting.hpp:184-290)
 * with SampleSplittersNumStringsPolicy and AllToAllStringImpl with
 * EmptyLcpByteEncoderMemCpy (mpi/alltoall.hpp:724-804): local sort; the
 * average LCP (getAvgLcp, misc.hpp:68-87); splitters from samples cut to
 * 200 (avg + 5) bytes (computePartition, misc.hpp:473-531;
 * samplingStrategies.hpp:25-55); whole strings exchanged and merged; the
 * output is every PE's received strings, whole and sorted, with LCPs (the
 * reference's returned StringLcpContainer).  As in the reference, p == 1 returns
 * the local sort (:230-232).  Byte-identical strings are indistinguishable in
 * this output; `source` orders them by (sender PE, local index).  One GPU
 * holds all PEs: the exchange and merge are a projection of one global sort. */
int dsss_ms_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                 const dsss_opts* opts, dsss_ms_result* out, dsss_stream_t stream);

/* Outputs of hQuicksort: the PEs' sorted strings back to back in rank order,
 * device arrays of n entries unless noted. */
typedef struct dsss_hq_result {
    uint64_t* counts;         /* HOST [p]: strings PE r holds after the sort */
    uint8_t* chars;           /* the output strings, each followed by a NUL */
    uint64_t chars_capacity;  /* bytes at chars: at least the sum of (length + 1) */
    uint64_t* offsets;        /* start of each output string in chars */
    uint32_t* lengths;        /* length of each output string */
    uint32_t* source;         /* optional: input index of each output string */
    uint32_t levels;          /* set by the call: hypercube levels (log2 of the largest power of two <= p) */
} dsss_hq_result;

/* RQuick::sort (src/sorter/RQuick/RQuick.hpp:1109-1115 -> :834-1104, sortRec
 * :415-627) as the hQuicksort executable runs it
 * (src/executables/HQuicksort.cpp:307-358: robust, StringComparator, PE r's
 * std::mt19937_64 seeded with seed + r; the executable passes 3469931): PEs
 * past the largest power of two hand their strings to PE r - 2^k, each PE
 * sorts, and every hypercube level splits each subcube at a pivot (one of the
 * subcube's first PE's two middle strings) with random tie-breaking and
 * exchanges halves with the partner PE.  The counts and the strings of every
 * PE are the reference's, bit for bit.  Byte-identical strings are
 * indistinguishable in this output; `source` names them in global order.
 * One GPU holds all PEs: the levels relabel string owners on one global sort
 * and the strings are written once. */
int dsss_hq_sort(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin, uint64_t seed,
                 dsss_hq_result* out, dsss_stream_t stream);

/* Batched form (no reference counterpart: the reference sorts one string set
 * per MPI job): nsets independent string sets of p PEs each in one arena, run
 * through one pipeline.  part_begin has nsets*p + 1 entries; PE q of set s
 * holds ids [part_begin[s*p + q], part_begin[s*p + q + 1]).  Each set's result
 * is exactly what dsss_pd_sort gives for that set alone: local_order holds
 * arena ids, perm_pe is the PE inside the set, and set s's merged sequences
 * fill the positions [part_begin[s*p], part_begin[(s+1)*p]) of perm_index,
 * perm_pe and merged_lcp.  intervals (HOST, nsets*p*p) and recv_counts (HOST,
 * nsets*p) hold the sets one after the other.  nsets*p <= 1024. */
int dsss_pd_sort_batched(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p,
                         const uint64_t* part_begin, const dsss_opts* opts, dsss_pd_result* out,
                         dsss_stream_t stream);
int dsss_pd_sort_batched_host(dsss_ctx* ctx, const dsss_arena* in, uint32_t nsets, uint32_t p,
                              const uint64_t* part_begin, const dsss_opts* opts, dsss_pd_result* out,
                              dsss_stream_t stream);

/* ---- stages (one per reference seam) ------------------------------------ */

/* tlx::sort_strings_detail::radixsort_CI3(StringLcpPtr, 0, 0)
 * (tlx/sort/strings/radix_sort.hpp:861-884), called per PE at prefix_doubling.hpp:228:
 * sorts each PE's strings, order[i] = input index, lcp[i] = LCP with i-1 in
 * the same PE (0 at each PE start). */
int dsss_local_sort_lcp(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                        const dsss_opts* opts, uint32_t* order, uint32_t* lcp, dsss_stream_t stream);

/* computeDistinguishingPrefixes<StringPtr, AllToAllHashesNaive>
 * (prefix_doubling.hpp:156-198) over BloomFilter::filter rounds
 * (bloomfilter.hpp:1415-1556): order/lcp are a local sort per PE (as
 * dsss_local_sort_lcp writes them); dp[i] is the DP length of the string at
 * local position i.  Exact 64-bit dedup of XXH64 prefix hashes mod 2^64-1,
 * depths 8, 24, 40, 72, ...  round_counts (host, may be NULL) receives the
 * candidate count after each round, up to max_rounds entries; *rounds the
 * number of rounds run. */
int dsss_dp_prefixes(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                     const uint32_t* order, const uint32_t* lcp, uint32_t* dp,
                     uint64_t* round_counts, uint32_t max_rounds, uint32_t* rounds,
                     dsss_stream_t stream);

/* One round of BloomFilter<…>::filter (bloomfilter.hpp:1415-1489 round 0,
 * :1491-1556 later rounds) over PEs whose strings are locally sorted
 * (order/lcp as dsss_local_sort_lcp writes them, every PE's first LCP 0):
 * candidates = ascending positions still undecided (NULL = every position,
 * the first round); results[c] = depth (or the length at EOS) for each
 * candidate (setDepth :1380-1411); next receives the positions that stay
 * candidates, *m_next their count (host). */
int dsss_dp_round(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, const uint32_t* lcp,
                  const uint32_t* candidates, uint64_t m, uint32_t depth, uint32_t* results, uint32_t* next,
                  uint64_t* m_next, dsss_stream_t stream);

/* XXHasher::hash(str, depth, UINT64_MAX) (bloomfilter.hpp:1094-1102) over
 * xxh::hash_state_t<64> (hash/xxhash.hpp:508-706) for strings ids[0..m):
 * hash[j] = XXH64(seed 0) of the first min(depth, len) bytes of string ids[j]
 * (the whole string when shorter), mod 2^64-1. */
int dsss_prefix_hash(const dsss_arena* in, const uint32_t* ids, uint64_t m, uint32_t depth,
                     uint64_t* hash, dsss_stream_t stream);

/* computePartition<Sampler>(ptr, 2, dp) (misc.hpp:531-587, indexed :650-708):
 * regular DP-truncated samples per PE, sorted, p-1 splitters, binary search
 * per PE.  order/dp as dsss_dp_prefixes uses them; intervals (HOST, p*p) as in
 * dsss_pd_result. */
int dsss_partition(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                   const uint32_t* order, const uint32_t* dp, const dsss_opts* opts,
                   uint64_t* intervals, dsss_stream_t stream);

/* AllToAllStringImplPrefixDoubling::alltoallv (mpi/alltoall.hpp:910-1008)
 * with EmptyPrefixDoublingLcpByteEncoderMemCpy (mpi/byte_encoder.hpp:139-171)
 * between p PEs of one GPU: builds every PE's receive container, back to
 * back in PE order.  Inputs: the local sort (local_order/lcp per PE, as
 * dsss_local_sort_lcp), dp in local order, intervals (HOST p*p, q*p + r).
 * Each string contributes bytes [lcp', dp) and a NUL, lcp' = 0 at the first
 * string of every interval (setLcpAtStartOfInterval :396-404).  Per received
 * string (device, n): recv_char_start (optional) its byte offset, recv_lcp
 * lcp', recv_index its index in the sender's local order, recv_pe the sender.
 * HOST outputs: *char_total, recv_char_begin[p+1] (optional),
 * recv_counts/recv_offsets [r*p + q] (optional): strings PE r got from q and
 * q's bucket offset.  recv_chars == NULL: sizes and per-string arrays only. */
int dsss_bucket_scatter(dsss_ctx* ctx, const dsss_arena* in, uint32_t p, const uint64_t* part_begin,
                        const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, const uint64_t* intervals,
                        uint8_t* recv_chars, uint64_t recv_capacity, uint64_t* char_total, uint64_t* recv_char_begin,
                        uint32_t* recv_char_start, uint32_t* recv_lcp, uint32_t* recv_index, uint32_t* recv_pe,
                        uint64_t* recv_counts, uint64_t* recv_offsets, dsss_stream_t stream);

/* choose_merge<AllToAllStringImplPrefixDoubling> (merging.hpp:66-123) with
 * LcpStringLoserTree_::writeElementsToStream(…, oldLcps)
 * (merge/bingmann-lcp_losertree.hpp:375-428), for nrecv receive containers
 * back to back (1 = one PE's container), each of p source runs:
 * recv_chars holds the prefix-compressed NUL-terminated strings,
 * recv_char_start (optional) their byte offsets, recv_lcp their sender-side
 * LCPs; recv_counts/recv_offsets (HOST, nrecv*p, [r*p + q]) the strings of
 * source q and q's bucket offset.  Outputs per merged position (device):
 * order = index into the containers, merged_lcp (0 at each PE start),
 * old_lcp (the sender-side LCP, 0 at run starts), perm_index/perm_pe (the
 * (stringIndex, PEIndex) tag); all but order optional.  Byte-identical
 * strings keep source order; the reference's loser tree orders them by
 * tournament history. */
int dsss_lcp_merge(dsss_ctx* ctx, const uint8_t* recv_chars, uint64_t char_bytes, const uint32_t* recv_char_start,
                   const uint32_t* recv_lcp, uint64_t n, uint32_t nrecv, uint32_t p, const uint64_t* recv_counts,
                   const uint64_t* recv_offsets, uint32_t* order, uint32_t* merged_lcp, uint32_t* old_lcp,
                   uint32_t* perm_index, uint32_t* perm_pe, dsss_stream_t stream);

/* The receiving side of DistributedMergeSort::sort
 * (lcp_aware_number_string_splitting.hpp:184-290) for PEs on several GPUs:
 * dsss_lcp_merge on receive containers of whole strings (sent with DP =
 * length), then every merged string whole — its prefix restored as
 * StringLcpContainer::extendPrefix does (strings/stringcontainer.hpp:248-333)
 * — NUL-terminated, back to back in merged order (out_offsets, out_lengths:
 * device, n each).  The output bytes are char_bytes + the sum of recv_lcp;
 * *out_bytes gets them, and DSSS_EINVAL when out_capacity is below them. */
int dsss_lcp_merge_strings(dsss_ctx* ctx, const uint8_t* recv_chars, uint64_t char_bytes,
                           const uint32_t* recv_char_start, const uint32_t* recv_lcp, uint64_t n, uint32_t nrecv,
                           uint32_t p, const uint64_t* recv_counts, const uint64_t* recv_offsets, uint32_t* order,
                           uint32_t* merged_lcp, uint8_t* out_chars, uint64_t out_capacity, uint64_t* out_offsets,
                           uint32_t* out_lengths, uint64_t* out_bytes, dsss_stream_t stream);

/* calc_lcp of sorted neighbours (strings/stringtools.hpp:158-166): lcp[i] =
 * LCP(string order[i-1], string order[i]) for i >= 1, lcp[0] = 0. */
int dsss_adjacent_lcp(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, uint64_t m, uint32_t* lcp,
                      dsss_stream_t stream);

/* No counterpart in the reference (which never runs on a GPU): dsss_adjacent_lcp
 * for callers that must not allocate device memory — code running inside
 * another framework's memory pool, where a raw cudaMalloc bypasses the pool
 * and can fail once the pool holds the free memory, and latency-critical
 * loops that cannot take the device-wide synchronisation of cudaMalloc /
 * cudaFree.  Same result as dsss_adjacent_lcp; no context, no allocation.
 * Its scratch is a static device array of 16 MiB + 256 B that every GPU
 * loading the library holds until the process exits, so m <= 4,194,304
 * strings per call (larger m returns DSSS_EINVAL).  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress) with the
 * device current; make that first call before any stream capture.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller. */
int dsss_adjacent_lcp_noalloc(const dsss_arena* in, const uint32_t* order, uint64_t m, uint32_t* lcp,
                              dsss_stream_t stream);

/* ---- PEs on several GPUs ---------------------------------------------------
 * One process per GPU, p_local PEs each (global PE ids q_first..); the caller
 * runs the collectives between these calls (NCCL through torch.distributed in
 * the Python package's dist.py).  Each entry is one piece of the reference's
 * distributed path around one of its exchanges.
 *
 * One BloomFilter::filter round on this GPU's sorted PEs (order/lcp as from
 * dsss_local_sort_lcp with the PE bounds): classification at depth (EOS, LCP
 * duplicates, roots, hashed: bloomfilter.hpp:1162-1227, 1273-1331), dp of every
 * candidate, state_out[i] = 1 for LCP duplicates and roots, and the positions
 * and XXH64 filter hashes of every hashed candidate (hpos, hval, *m of them,
 * in position order).  state_in NULL: the first round (all candidates). */
int dsss_dp_classify_hash(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* order, const uint32_t* lcp,
                          const uint8_t* state_in, uint32_t depth, uint32_t* dp, uint8_t* state_out, uint32_t* hpos,
                          uint64_t* hval, uint64_t* m, dsss_stream_t stream);
/* Groups (hval, hpos) by owning GPU, equal slices of the hash range as
 * SendOnlyHashesToFilter::sendToFilter (bloomfilter.hpp:581-640) cuts it;
 * counts (HOST, nowner): the group sizes, in owner order. */
int dsss_hash_route(dsss_ctx* ctx, const uint64_t* hval, const uint32_t* hpos, uint64_t m, uint32_t nowner,
                    uint64_t* out_hval, uint32_t* out_hpos, uint64_t* counts, dsss_stream_t stream);
/* The round's hash records in hash order, stable: ips4o::sort of the
 * HashStringIndex records (bloomfilter.hpp:1512), which the Golomb-coded
 * exchange needs (each destination's hashes ascending).  Since the owner of a
 * hash is monotone in it, the sorted records are also grouped by owner. */
int dsss_hash_sort(dsss_ctx* ctx, const uint64_t* hval, const uint32_t* hpos, uint64_t m, uint64_t* out_hval,
                   uint32_t* out_hpos, dsss_stream_t stream);
/* Owner side of FindDuplicates::findDuplicates (bloomfilter.hpp:662-765):
 * dup[j] = 1 iff hval[j] occurs at least twice among the m received hashes. */
int dsss_hash_dups(dsss_ctx* ctx, const uint64_t* hval, uint64_t m, uint8_t* dup, dsss_stream_t stream);
/* state[hpos[j]] = 1 where dup[j] (the duplicates returned to their senders,
 * bloomfilter.hpp:767-817); *candidates = positions with state 1. */
int dsss_dp_apply(dsss_ctx* ctx, const uint32_t* hpos, const uint8_t* dup, uint64_t m, uint8_t* state, uint64_t n,
                  uint64_t* candidates, dsss_stream_t stream);
/* Packs strings ids[j] truncated to min(length, trunc[j]) (trunc NULL: whole)
 * back to back with a NUL each (the splitter sample, samplingStrategies.hpp:
 * 57-89); out_offsets/out_lengths (device, m); *bytes the packed size;
 * out_chars NULL: sizes only. */
int dsss_pack_strings(dsss_ctx* ctx, const dsss_arena* in, const uint32_t* ids, const uint32_t* trunc, uint64_t m,
                      uint8_t* out_chars, uint64_t capacity, uint64_t* out_offsets, uint32_t* out_lengths,
                      uint64_t* bytes, dsss_stream_t stream);
/* compute_interval_binary (misc.hpp:376-414) of this GPU's p_local PEs against
 * splitters->n <= p_global - 1 splitters gathered from every GPU; intervals
 * (HOST, p_local x p_global).  indexed: spl_index (HOST) the splitters' global
 * indices and pe_index (HOST, p_local) the global index of each local PE's
 * first string (indexStringCompare, misc.hpp:335-345). */
int dsss_partition_search(dsss_ctx* ctx, const dsss_arena* in, uint32_t p_local, const uint64_t* part_begin,
                          const uint32_t* local_order, const dsss_arena* splitters, const uint64_t* spl_index,
                          uint32_t p_global, const uint64_t* pe_index, int indexed, uint64_t* intervals,
                          dsss_stream_t stream);
/* Sender side of AllToAllStringImplPrefixDoubling::alltoallv (alltoall.hpp:
 * 910-1008): the receive container of every one of the p_global PEs, from this
 * GPU's senders, back to back (bytes [lcp', dp) + NUL per string); per string
 * char_start (relative to its receiver's container) and the sent LCP;
 * recv_char_begin (HOST, p_global + 1), counts/offsets (HOST, [r*p_local + q]). */
int dsss_bucket_send(dsss_ctx* ctx, const dsss_arena* in, uint32_t p_local, const uint64_t* part_begin,
                     const uint32_t* local_order, const uint32_t* lcp, const uint32_t* dp, uint32_t p_global,
                     uint32_t q_first, const uint64_t* intervals, uint8_t* send_chars, uint64_t capacity,
                     uint64_t* char_total, uint64_t* recv_char_begin, uint32_t* char_start, uint32_t* send_lcp,
                     uint64_t* counts, uint64_t* offsets, dsss_stream_t stream);
/* Receiver side: copies blocks (HOST, nblocks x {src string, dst string,
 * strings, src byte, dst byte, bytes}) of received containers into receiver
 * order; dst_start = src_start + the block's dst byte. */
int dsss_regroup(dsss_ctx* ctx, uint32_t nblocks, const uint64_t* blocks, const uint8_t* src_chars,
                 uint8_t* dst_chars, const uint32_t* src_start, uint32_t* dst_start, const uint32_t* src_lcp,
                 uint32_t* dst_lcp, uint64_t n, dsss_stream_t stream);

/* ---- request server (no reference counterpart) ---------------------------
 * Continuous batching of independent sort requests onto one GPU.  Requests
 * (host arenas, p PEs each) are queued on submit; worker threads, each with
 * its own stream, take the requests at the head of the queue that fit one
 * batch and the device-memory budget and run them as one
 * dsss_pd_sort_batched call, several batches in flight at once.  Device
 * memory comes from a pool that keeps freed blocks resident up to the budget;
 * a batch is admitted only if its exact footprint (arena, outputs, pipeline
 * scratch) fits beside the batches in flight.  Each request's result equals
 * dsss_pd_sort_host on that request alone.  Input and output host buffers
 * must stay valid until dsss_server_wait returns for the ticket. */
typedef struct dsss_server dsss_server;

typedef struct {
    int device;
    uint32_t workers;           /* batches in flight at once; 0 -> 2 */
    uint32_t p;                 /* PEs per request (1..1024) */
    uint32_t max_sets;          /* requests per batch; 0 -> 1024 / p (also capped there) */
    uint64_t max_batch_strings; /* strings per batch beyond its first request; 0 -> no limit */
    uint64_t hbm_budget;        /* device bytes the server may hold; 0 -> 150e9 */
    dsss_opts opts;
    uint32_t flags;             /* DSSS_SERVER_* */
    uint64_t reserve_bytes;     /* device memory mapped into the pool at start (kept resident) */
} dsss_server_config;

/* Record t_copied (one extra stream synchronisation per batch). */
#define DSSS_SERVER_TIMESTAMPS 1u

typedef struct {
    int status;                 /* DSSS_OK or the batch's error */
    uint32_t batch_sets;        /* requests in the batch this one ran in */
    uint64_t batch_id;
    uint64_t batch_strings;
    double t_submit, t_admit, t_done; /* seconds, dsss_clock_now() */
    double t_copied, t_sorted;        /* batch inputs on the device; batch sorted */
    char error[160];
} dsss_request_stats;

typedef struct {
    uint64_t queued;
    uint64_t reserved_bytes;     /* footprints of the batches in flight */
    uint64_t max_reserved_bytes; /* the most ever reserved at once (<= hbm_budget) */
    uint64_t batches;
    uint64_t batched_requests;
    uint64_t hbm_budget;
} dsss_server_info_t;

double dsss_clock_now(void);
int dsss_server_create(const dsss_server_config* cfg, dsss_server** out);
/* part_begin: p + 1 PE bounds of the request, or NULL for p equal slices.
 * out: host arrays as for dsss_pd_sort_host. */
int dsss_server_submit(dsss_server* s, const dsss_arena* in, const uint64_t* part_begin, dsss_pd_result* out,
                       uint64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit; DSSS_ETIMEDOUT keeps the
 * ticket valid), fills stats and releases the ticket; returns its status. */
int dsss_server_wait(dsss_server* s, uint64_t ticket, int64_t timeout_ms, dsss_request_stats* stats);
int dsss_server_info(dsss_server* s, dsss_server_info_t* info);
/* Device bytes a request of n strings and char_bytes bytes needs alone. */
uint64_t dsss_server_footprint(dsss_server* s, uint64_t n, uint64_t char_bytes);
/* Finishes every queued request, then stops the workers. */
int dsss_server_destroy(dsss_server* s);

/* ---- synthetic inputs (host) --------------------------------------------- */

/* distribute_strings (src/mpi/readInput.hpp:40-104) for p PEs held by one
 * GPU: the file's first S = min(size, max_size) bytes (max_size 0: all) in p
 * byte slices (the first S % p one byte longer); every '\n' becomes a NUL;
 * PE r > 0 starts just after the first '\n' of its slice (its first line goes
 * to PE r - 1, as the reference's shift does); a NUL closes the file when it
 * does not end with one.  file: host bytes.  Writes *char_bytes (S, + 1 for
 * the closing NUL) and, when chars != NULL: chars (device, chars_cap >=
 * char_bytes + 32, the tail zeroed), offsets / lengths (device, cap_n entries)
 * of the *n lines in file order, part_begin (HOST, p + 1 line indices): an
 * arena ready for dsss_pd_sort / dsss_ms_sort.  Where the reference reads
 * past a buffer it is an error: a slice of PE r > 0 without a '\n', or fewer
 * bytes than PEs (an empty last slice). */
int dsss_distribute_lines(dsss_ctx* ctx, const uint8_t* file, uint64_t size, uint64_t max_size, uint32_t p,
                          uint8_t* chars, uint64_t chars_cap, uint64_t* offsets, uint32_t* lengths, uint64_t cap_n,
                          uint64_t* n, uint64_t* char_bytes, uint64_t* part_begin, dsss_stream_t stream);

/* Varint coding of LCP arrays, the wire format of the string exchange with
 * compressLcps (sendLcps, src/mpi/alltoall.hpp:406-425; Writer::PutVarint,
 * src/encoding/integer_compression.hpp:66-140: 7 bits per byte, least
 * significant first, the high bit on every byte but the last).
 * encode: values (device, n) to out (device, out_cap bytes); *out_bytes = the
 * coded size (out == NULL: size query only); ranges [range_begin[r],
 * range_begin[r+1]) (HOST, nranges + 1 value indices) get their byte counts
 * in range_bytes (HOST, nranges), as IntegerCompression::writeRanges
 * (src/mpi/byte_encoder.hpp:31-53) reports them.
 * decode: nbytes coded bytes (device) holding exactly n values (device out);
 * a cut-off, over-long or too large value is an error. */
int dsss_varint_encode(dsss_ctx* ctx, const uint32_t* values, uint64_t n, const uint64_t* range_begin,
                       uint32_t nranges, uint8_t* out, uint64_t out_cap, uint64_t* out_bytes, uint64_t* range_bytes,
                       dsss_stream_t stream);
int dsss_varint_decode(dsss_ctx* ctx, const uint8_t* in, uint64_t nbytes, uint32_t* values, uint64_t n,
                       dsss_stream_t stream);

/* Golomb/delta coding of sorted 64-bit values, the wire format of the hash
 * exchange with sequentialGolombEncoding (AllToAllHashesGolomb,
 * src/sorter/distributed/bloomfilter.hpp:164-313, over getDeltaEncoding /
 * getDeltaDecoding, src/encoding/golomb_encoding.hpp:50-110, and thrill's
 * GolombBitStreamWriter / Reader, src/encoding/golomb_bit_stream.hpp).  A
 * range of c > 0 ascending values becomes the block [S, b, v_0, bit words]
 * (S = words after S); the bit words hold, most significant bit first, each
 * gap v_i - v_{i-1} as q = gap / b ones, a zero and gap mod b in truncated
 * binary; the unused bits of the last word are ones.  An empty range takes
 * no words.
 * param: getB(max_value, count) (golomb_encoding.hpp:50-59); param_hashes:
 * the hash exchange's b for count hashes sent to one of p PEs
 * (bloomfilter.hpp:194-197: getB over 2^64 - 1 / p, 1 replaced by 2e10).
 * encode: values (device) in nranges ranges of range_counts[r] values (HOST),
 * parameters b[r] (HOST, >= 1) into out (device, out_cap words);
 * *out_words = the total and range_words[r] (HOST) each range's words
 * (out == NULL: size query only).  Values must ascend inside a range; a gap
 * of more than 2^31 b is rejected.
 * decode: nwords words (device) of back-to-back blocks, read block after
 * block as the receiving PE does (bloomfilter.hpp:230-242); *n_values values
 * to values (device, cap_values; NULL: size query), block_counts[j] (HOST,
 * max_blocks) the values of block j, *nblocks the blocks. */
uint64_t dsss_golomb_param(uint64_t max_value, uint64_t count);
uint64_t dsss_golomb_param_hashes(uint64_t count, uint32_t p);
int dsss_golomb_encode(dsss_ctx* ctx, const uint64_t* values, const uint64_t* range_counts, uint32_t nranges,
                       const uint64_t* b, uint64_t* out, uint64_t out_cap, uint64_t* out_words, uint64_t* range_words,
                       dsss_stream_t stream);
int dsss_golomb_decode(dsss_ctx* ctx, const uint64_t* words, uint64_t nwords, uint64_t* values, uint64_t cap_values,
                       uint64_t* n_values, uint64_t* block_counts, uint32_t max_blocks, uint32_t* nblocks,
                       dsss_stream_t stream);

/* D/N-ratio strings (the role of DNRatioGenerator, util/random_string_generator.hpp:166-318),
 * seeded and reproducible: string i is (k - d) 'A's, the d base-26 digits
 * ('A' = 0) of pi(i) for a seeded permutation pi of [0, n), then uniform
 * 'A'-'Z' up to its length; d = ceil(log26 n).  A seeded fraction frac_long of
 * the strings uses (len_long, k_long) instead of (len_short, k_short).
 * Layout: strings back to back, each followed by one NUL.
 * Call with chars == NULL to get *char_bytes only. */
int dsss_gen_dn(uint64_t n, uint32_t len_short, uint32_t k_short, uint32_t len_long, uint32_t k_long,
                double frac_long, uint64_t seed, uint8_t* chars, uint64_t* offsets, uint32_t* lengths,
                uint64_t* char_bytes);

/* Text over {A,C,G,T} from a seeded order-3 Markov source; each position the
 * source emits starts, with probability copy_prob, a copy of 1-4 KiB from an
 * earlier offset.  text gets text_len bytes. */
int dsss_gen_markov_text(uint64_t text_len, double copy_prob, uint64_t seed, uint8_t* text);

/* All suffixes of a text of text_len bytes, truncated to max_len bytes:
 * offsets[i] = i, lengths[i] = min(max_len, text_len - i). */
int dsss_gen_suffixes(uint64_t text_len, uint32_t max_len, uint64_t* offsets, uint32_t* lengths);

/* One serving request: n strings, lengths Zipf(s) on [min_len, max_len],
 * bytes uniform 0x21-0x7E after a shared per-request prefix of length
 * uniform in [0, len/2].  Layout as dsss_gen_dn. */
int dsss_gen_request(uint64_t n, uint32_t min_len, uint32_t max_len, double zipf_s, uint64_t seed,
                     uint8_t* chars, uint64_t* offsets, uint32_t* lengths, uint64_t* char_bytes);

/* The same generators writing device memory, so that a configuration's input
 * never crosses PCIe (the reference's generators build each PE's strings in
 * place, util/random_string_generator.hpp:167-318, :432-509).  Byte for byte
 * the host generators' output; chars, offsets and lengths are device
 * pointers (chars 16-byte aligned), the call is asynchronous on `stream`
 * except for the read-back of the total.  chars == NULL: *char_bytes only.
 * Errors: DSSS_EINVAL (arguments, n >= 2^32), DSSS_ENOMEM (scratch). */
int dsss_gen_dn_dev(dsss_ctx* ctx, uint64_t n, uint32_t len_short, uint32_t k_short, uint32_t len_long,
                    uint32_t k_long, double frac_long, uint64_t seed, uint8_t* chars, uint64_t* offsets,
                    uint32_t* lengths, uint64_t* char_bytes, dsss_stream_t stream);
int dsss_gen_suffixes_dev(uint64_t text_len, uint32_t max_len, uint64_t* offsets, uint32_t* lengths,
                          dsss_stream_t stream);
int dsss_gen_request_dev(dsss_ctx* ctx, uint64_t n, uint32_t min_len, uint32_t max_len, double zipf_s,
                         uint64_t seed, uint8_t* chars, uint64_t* offsets, uint32_t* lengths, uint64_t* char_bytes,
                         dsss_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DSSS_H */
