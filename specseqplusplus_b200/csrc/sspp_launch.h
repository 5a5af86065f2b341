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
// lows: also the lowest rows and leftmost columns (the first init pass);
// assigned: recorded once perm / newidx / dim are written (before the columns
// are scattered), or null
int reorder(Device& D, bool lows, cudaStream_t s, cudaEvent_t assigned = nullptr);
int64_t reorder_total_slot(const Device& D);  // index into D.blk of the arena total

// per-complex slice starts (k+1 each) of the sorted pairs and essentials
int batch_bounds(int32_t k, const int64_t* d_cstart, int64_t npairs, const int64_t* pairs, int64_t ness,
                 const int64_t* ess, int64_t* d_pstart, int64_t* d_estart, cudaStream_t s);
// pairs / essentials with each complex's first column subtracted
int batch_localize(int64_t npairs, int64_t ness, int32_t k, const int64_t* d_cstart, const int64_t* pairs,
                   const int64_t* ess, int64_t* lpairs, int64_t* less, cudaStream_t s);

// lows_done: the reorder computed the lowest rows and leftmost columns
int init_passes(Device& D, bool lows_done, cudaStream_t s);
// keep_rows: leave negative rows in the columns (whole reduced columns, for
// representative cycles); otherwise they are removed.
// final (no dualization follows): also the inline apparent columns (as
// build_apparent) and the per-dimension row bounds (as active_list)
// columns [cb, ce) (ce < 0: to the end); reset: clear the row bounds first
// (the first of the launches that together cover every column)
int init_compress(Device& D, const uint8_t* dropped, bool keep_rows, bool final, cudaStream_t s, int64_t cb = 0,
                  int64_t ce = -1, bool reset = true);
// rows_done: init_compress already gathered the row bounds
int active_list(Device& D, bool rows_done, cudaStream_t s);
// D.app from the pivot table as it stands (apparent pairs only)
int build_apparent(Device& D, cudaStream_t s);
// anti-transpose of the compressed matrix behind the primal columns in the
// arena; remaps pivots, states, dims and the per-dimension column ranges.
// mode 1: the whole matrix; mode 2: after the edge columns were reduced (the
// 0-dimensional pairs are final, the vertices' dual columns are skipped)
int dualize(Device& D, int mode, cudaStream_t s);
int extract_pairs(Device& D, int dual, const uint8_t* dropped, cudaStream_t s);

// Device work queue of (complex, block) items (one persistent launch per
// schedule; see k_reduce_queue).  An item is one spectral-sequence block of
// one complex in one dimension: the slice of the active list it adds to the
// window and the band's lowest row.
struct QItem {
    int32_t cplx;
    int32_t nbeg, nend;  // active-list entries that enter the window with this block
    int32_t minrow;      // the band's lowest row (INT32_MIN: the dimension's completion sweep)
    int32_t flags;       // QF_* below
    int32_t pad[3];
};
enum : int32_t {
    QF_LAST_OF_DIM = 1,  // the complex's next item (if any) is of its next dimension
    QF_HALF = 2,         // this item reads the parked columns from the second half of its complex's list
};

struct QueueArgs {
    const QItem* items;
    int32_t nitems, ncplx;
    int* taken;            // [nitems] entries handed out
    int* done;             // [nitems] entries finished
    int* lin;              // [nitems + 1] parked columns each item starts with (written by its predecessor)
    int* cur;              // [ncplx] current item of each complex; -1 once the complex is finished
    int* gate;             // [ncplx] 1: the complex's block sequence waits for its CTA-tier columns
    int* hpend;            // [ncplx] CTA-tier columns of the complex not finished yet
    const int32_t* item_end;   // [ncplx] one past the complex's last item
    const int64_t* list_off;   // [ncplx] the complex's parked-column list (two halves)
    const int32_t* list_cap;   // [ncplx] entries per half
    int2* lists;           // (column, lowest row)
    int32_t* pool;         // deferred columns for the CTA tier (-1 until written)
    int32_t* pool_c;       // their complexes
    int32_t pool_cap;
    int* pool_head;        // next slot the CTA tier takes
    int* pool_tail;        // next slot written
    int* finished;         // complexes finished
    int* abort;            // set on any failure: every block leaves
    int32_t heavy_ctas;    // blocks [0, heavy_ctas) reduce CTA-tier columns; the others run warps
    int32_t gate_left;     // a complex's next dimension starts once at most this many of its CTA-tier columns are left
    int32_t chunk;         // entries a warp takes at a time
    int32_t cap1;          // warp buffers (ints)
    long long spin_limit;  // idle polls before a block gives up (SSPP_ERR_TIMEOUT)
};

// per complex: active columns and band bounds of each dimension, from the
// state after the init passes (out: [k][kNumDims] each)
int queue_complex_info(const Device& D, int32_t k, const int64_t* d_cstart, int32_t* act_cnt, int32_t* min_row,
                       int32_t* max_row, cudaStream_t s);
// blocks per SM of the queue kernel with these capacities (0: it does not fit)
cudaError_t queue_configure(int cap1, int cap2, int threads, int* blocks_per_sm);
// cooperative launch of the queue kernel on `grid` blocks
cudaError_t reduce_queue_launch(const Device& D, int cap1, int cap2, int threads, const QueueArgs& Q, int grid,
                                cudaStream_t s);

cudaError_t reduce_configure(int cap1, int cap2, int heavy_threads, int* light_blocks_per_sm,
                             int* heavy_blocks_per_sm);
// ctr: the step's 8 counters; the launch's last block also marks the step's
// CTA-tier pool slice (ctr[2], and ctr_next[1] of the next step when given)
void reduce_light_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                         int chunk, int* ctr, int* ctr_next, int grid, cudaStream_t s);
// The same step in two launches: k_light_filter lists the window's runnable
// columns (active[beg, end)) in D.runlist, then the warp tier takes them
// `chunk` at a time.
void reduce_light_filtered_launch(const Device& D, int32_t beg, int32_t end, int32_t minrow, int cap, int chunk,
                                  int* ctr, int* ctr_next, int filter_grid, int grid, cudaStream_t s);
void reduce_heavy_launch(const Device& D, int cap, int threads, int* ctr, int grid, cudaStream_t s);

}  // namespace sspp
