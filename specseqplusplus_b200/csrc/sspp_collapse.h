// Flag-complex edge collapse (model bit 2): scratch buffers and launcher.
#pragma once
#include <cuda_runtime.h>

#include "sspp_internal.h"

namespace sspp {

struct CollapseScratch {
    int32_t* eu = nullptr;       // [E] edge endpoints (vertex = reordered column index), eu < ev
    int32_t* ev = nullptr;
    int32_t* ecol = nullptr;     // [E] reordered column of edge e
    int32_t* deg = nullptr;      // [nv + 1] degrees, then fill cursors
    int64_t* adj_off = nullptr;  // [nv + 1]
    uint64_t* adj = nullptr;     // [2E] (neighbour << 32 | edge id), ascending per vertex
    uint8_t* arr = nullptr;      // [E] arrival test: 0 dominated, 1 kept, 2 kept with triangles to re-examine
    uint8_t* crit = nullptr;     // [E] critical (kept) edges
    uint8_t* ins = nullptr;      // [E] in the re-examination set
    int32_t* heap = nullptr;     // [E] re-examination set, max-heap
    int32_t* cas = nullptr;      // [E] arrivals with re-examinations, ascending
    int32_t* open = nullptr;     // [E * kOpen] per arrival: its triangles' edges dominated at their arrival
    int8_t* nopen = nullptr;     // [E] how many (-1: more than kOpen, or not listed)
    int32_t* cbuf = nullptr;     // overflow buffers of the common neighbourhoods
    int32_t* misc = nullptr;     // [8] device scalars
    int4* erec = nullptr;        // [E] neighbour-list bounds of both endpoints {off[u], off[u+1], off[v], off[v+1]}
    int2* vrec = nullptr;        // [nv] neighbour-list bounds {off[w], off[w+1]}
    int32_t* spec = nullptr;     // speculative cascade records, one per arrival with re-examinations
    int32_t* first_mark = nullptr;  // [nv] smallest record index keeping an edge at the vertex
    uint32_t* dirty_words = nullptr;  // [nv / 32] vertices of edges the applied records keep
    int64_t cap_e = 0, cap_v = 0, cap_cbuf = 0, cap_spec = 0;
};

// Marks dropped[] (reordered numbering) for the edges the collapse removes and
// every higher simplex with a removed facet, then empties those columns.
// Synchronises the stream twice (edge count, maximum degree).  Returns the
// number of kernels launched, or -1 with *err_msg on failure.
int collapse(Device& D, const DimInfo& info, uint8_t* dropped, CollapseScratch& S, cudaStream_t s,
             const char** err_msg);

void collapse_free(CollapseScratch& S);

}  // namespace sspp
