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
// Each launcher returns the number of kernels it launched.
int validate(Device& D, cudaStream_t s);  // sets ERRB_BAD_INPUT
// k complexes copied side by side (cstart/estart: k+1 column / entry starts on
// the device): shifts each one's face indices and col_ptr entries; *d_bad = 1
// when a face index lies outside its own complex
int batch_rebase(int64_t n, int64_t nnz, int32_t k, const int64_t* d_cstart, const int64_t* d_estart,
                 int64_t* colptr, int32_t* rows, int* d_bad, cudaStream_t s);
int reorder(Device& D, cudaStream_t s);
int64_t reorder_total_slot(const Device& D);  // index into D.blk of the arena total

// per-complex slice starts (k+1 each) of the sorted pairs and essentials
int batch_bounds(int32_t k, const int64_t* d_cstart, int64_t npairs, const int64_t* pairs, int64_t ness,
                 const int64_t* ess, int64_t* d_pstart, int64_t* d_estart, cudaStream_t s);
// pairs / essentials with each complex's first column subtracted
int batch_localize(int64_t npairs, int64_t ness, int32_t k, const int64_t* d_cstart, const int64_t* pairs,
                   const int64_t* ess, int64_t* lpairs, int64_t* less, cudaStream_t s);

int init_passes(Device& D, cudaStream_t s);
// keep_rows: leave negative rows in the columns (whole reduced columns, for
// representative cycles); otherwise they are removed.
int init_compress(Device& D, const uint8_t* dropped, bool keep_rows, cudaStream_t s);
int active_list(Device& D, cudaStream_t s);
// D.app from the pivot table as it stands (apparent pairs only)
int build_apparent(Device& D, cudaStream_t s);
// anti-transpose of the compressed matrix behind the primal columns in the
// arena; remaps pivots, states, dims and the per-dimension column ranges.
// mode 1: the whole matrix; mode 2: after the edge columns were reduced (the
// 0-dimensional pairs are final, the vertices' dual columns are skipped)
int dualize(Device& D, int mode, cudaStream_t s);
int extract_pairs(Device& D, int dual, const uint8_t* dropped, cudaStream_t s);

cudaError_t reduce_configure(int cap1, int cap2, int heavy_threads, int* light_blocks_per_sm,
                             int* heavy_blocks_per_sm);
void reduce_light_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                         int chunk, int* ctr, int grid, cudaStream_t s);
void heavy_slice_mark(const Device& D, int* ctr_k, int* ctr_next, cudaStream_t s);
void reduce_heavy_launch(const Device& D, int cap, int threads, int* ctr, int grid, cudaStream_t s);

}  // namespace sspp
