// High-dimension guided clearing: scratch buffers and launcher.
#pragma once
#include <cuda_runtime.h>

#include "sspp_internal.h"

namespace sspp {

struct HighclearScratch {
    int32_t* tup[kNumDims] = {};   // vertex tuples of dims 1..top, (d+1) ints per column
    int64_t cap_tup[kNumDims] = {};
    int32_t* deg = nullptr;         // [nv + 1]
    int64_t* adj_off = nullptr;     // [nv + 1]
    int32_t* adj = nullptr;         // [2 E]
    int32_t* adj_src = nullptr;     // [2 E] the vertex whose list holds each entry
    uint64_t* nmask = nullptr;      // [2 E] per entry (a, b): which candidates of a are neighbours of b
    int32_t* table = nullptr;       // open addressing, mask + 1 slots
    uint32_t mask = 0;
    int64_t* blk = nullptr;         // block sums of its own scans (the branch runs beside the reorder's scans)
    int64_t cap_deg = 0, cap_adj_off = 0, cap_adj = 0, cap_table = 0, cap_src = 0, cap_nmask = 0, cap_blk = 0;
};

// Up to this many candidates per simplex (max_iteration) the test runs on
// per-neighbour candidate masks, one thread per simplex; beyond, a group of
// lanes per simplex searches the neighbour lists.
constexpr int kMaskCandidates = 64;

// Sets cleared[] for the top-dimension columns the test proves positive;
// returns the number of kernels launched.  Buffers must be sized by the caller.
// from_input: the vertex tuples are read from the input matrix through
// D.perm / D.newidx (which is all it needs of the reorder: it can run beside
// the column scatter); otherwise from the reordered columns.
int highclear(Device& D, const DimInfo& info, int max_iteration, const uint8_t* dropped, HighclearScratch& S,
              cudaStream_t s, bool from_input = false);

}  // namespace sspp
