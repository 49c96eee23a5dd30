// Splitter sampling and partitioning (K5); see partition.cu.
#pragma once
#include "internal.cuh"
#include "strsort.cuh"

namespace dsss {

struct PartitionLayout {
    uint64_t cap;
    uint64_t* sample_lp;
    uint64_t* soff;
    uint32_t* slen;
    uint32_t* sorted;
    uint32_t* slcp;
    uint64_t* spl_off;
    uint32_t* spl_len;
    uint64_t* spl_index;
    uint64_t* pos;
    uint64_t* pb;
    uint32_t* set_nspl;
    SortLayout sort;
};

void layout_partition(Carve& c, PartitionLayout& L, uint64_t n, uint32_t p, uint32_t factor, uint32_t nsets = 1);

// local_order: per PE the string ids in sorted order; dp: their distinguishing
// prefixes (same positions).  intervals (host, p*p): strings PE q sends to PE r.
int partition_pes(const PartitionLayout& L, Ctx* ctx, const ArenaDev& a, uint32_t p, const uint64_t* pb,
                  const uint32_t* local_order, const uint32_t* dp, uint32_t sampler, uint32_t factor,
                  uint64_t* intervals, cudaStream_t st);

// The same for nsets independent sets of p PEs each: PE q of set s is
// pb[s*p + q] .. pb[s*p + q + 1]; intervals (host, nsets*p*p) per set as above.
int partition_sets(const PartitionLayout& L, Ctx* ctx, const ArenaDev& a, uint32_t nsets, uint32_t p,
                   const uint64_t* pb, const uint32_t* local_order, const uint32_t* dp, uint32_t sampler,
                   uint32_t factor, uint64_t* intervals, cudaStream_t st);

// PEs on several GPUs: intervals (host, p_local x p_global) of this GPU's
// p_local PEs against the nspl = sp.n <= p_global - 1 splitters in arena sp
// (gathered from every GPU).  Indexed compare: goff_host[g] is the global
// index of local PE g's first string, spl_index_host[k] the splitter's.
int partition_search(Ctx* ctx, const ArenaDev& a, uint32_t p_local, const uint64_t* pb, const uint32_t* local_order,
                     const ArenaDev& sp, const uint64_t* spl_index_host, uint32_t p_global, const uint64_t* goff_host,
                     int indexed, uint64_t* intervals, cudaStream_t st);

}  // namespace dsss
