// Host-side launchers of the engine's device passes.
#pragma once
#include <cuda_runtime.h>

#include "sspp_internal.h"

namespace sspp {

void fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t s);
void fill_i64(int64_t* p, int64_t v, int64_t n, cudaStream_t s);

// input (filtration order) -> dimension-sorted padded arena layout; writes
// D.newidx, D.perm, D.dim, D.desc, D.diminfo->col_begin/col_end; D.blk[scan
// total] holds the arena ints used.
void validate(Device& D, cudaStream_t s);  // sets ERRB_BAD_INPUT
void reorder(Device& D, cudaStream_t s);
int64_t reorder_total_slot(const Device& D);  // index into D.blk of the arena total

void init_passes(Device& D, cudaStream_t s);
void init_compress(Device& D, const uint8_t* dropped, cudaStream_t s);
void active_list(Device& D, cudaStream_t s);
void extract_pairs(Device& D, int dual, const uint8_t* dropped, cudaStream_t s);

int reduce_smem_bytes(int cap);
cudaError_t reduce_configure(int cap, int* blocks_per_sm);
void reduce_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                   int* chunk_ctr, int grid, cudaStream_t s);

}  // namespace sspp
