// Internal types shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sspp.h"

namespace sspp {

constexpr int kMaxDim = 7;          // dimensions 0..7 (the reference's MAXDIM is 5, include/bupt.h:48)
constexpr int kNumDims = kMaxDim + 1;

// Column states (one byte per column).
enum : uint8_t {
    ST_ACTIVE = 0,   // needs (more) reduction
    ST_OWNER = 1,    // owns the pivot at its lowest row
    ST_ZERO = 2,     // reduced to zero (positive) or empty input column
    ST_CLEARED = 3,  // zeroed by clearing (positive), never reduced
    ST_DROPPED = 4,  // removed by edge collapse
    ST_HEAVY = 5,    // handed from the warp tier to the CTA tier
};

// A column version occupies an arena slot at a 16-byte aligned offset: a
// 16-byte header {length, column, 0, 0} followed by the sorted row indices,
// padded with INT32_MAX to a multiple of four ints.  A column's descriptor
// packs (slot offset in ints << 24) | length.
constexpr int kLenBits = 24;
constexpr uint64_t kLenMask = (1ull << kLenBits) - 1;
constexpr int64_t kMaxColLen = int64_t(kLenMask);
constexpr int kHdr = 4;  // header ints
__host__ __device__ inline uint64_t pack_desc(uint64_t off, uint32_t len) { return (off << kLenBits) | len; }
__host__ __device__ inline uint64_t desc_off(uint64_t d) { return d >> kLenBits; }
__host__ __device__ inline uint32_t desc_len(uint64_t d) { return uint32_t(d & kLenMask); }
__host__ __device__ inline int64_t pad4(int64_t x) { return (x + 3) & ~int64_t(3); }
__host__ __device__ inline int64_t slot_ints(int64_t len) { return kHdr + pad4(len); }

// Pivot table entry of a row: the owning column (31 bits) and the arena slot
// of the owner's version (in 16-byte units, 33 bits), so a reader reaches the
// owner's entries with one dependent load.  No owner = all ones, which reads
// as a column index larger than any column.
constexpr uint64_t kNoOwner = ~0ull;
__host__ __device__ inline uint64_t pv_pack(int32_t col, uint64_t slot_off_ints) {
    return ((slot_off_ints >> 2) << 31) | uint64_t(uint32_t(col));
}
__host__ __device__ inline int32_t pv_col(uint64_t e) { return int32_t(e & 0x7fffffffu); }
__host__ __device__ inline uint64_t pv_slot(uint64_t e) { return (e >> 31) << 2; }  // slot offset in ints

// Error word bits set by kernels (device int).
enum : int {
    ERRB_BAD_INPUT = 1,
    ERRB_CAPACITY = 2,
    ERRB_TIMEOUT = 4,
    ERRB_LEN = 8,       // a column exceeded kMaxColLen
    ERRB_CHECK = 16,    // a self-check of the reduction failed (bad index skipped)
};

// Per-dimension summary after the init passes (in reordered numbering).
struct DimInfo {
    int32_t col_begin[kNumDims];   // reordered columns of dim d: [col_begin, col_end)
    int32_t col_end[kNumDims];
    int32_t act_begin[kNumDims];   // active list segment of dim d
    int32_t act_end[kNumDims];
    int32_t min_row[kNumDims];     // min first row over non-empty columns (DimMinRow)
    int32_t max_row[kNumDims];     // max low + 1 over active columns (DimMaxRow)
};

// Device counters (int64 each), reset at the start of a run.
enum CounterIdx {
    CNT_ADDITIONS = 0,
    CNT_ADD_INTS,
    CNT_PUBLISHED,
    CNT_DISPLACED,
    CNT_APPARENT,
    CNT_CLEARED,
    CNT_HIGHCLEAR,
    CNT_DROPPED,
    CNT_ACTIVE,
    CNT_NPAIRS,
    CNT_NESS,
    CNT_HEAVY_ADDS,  // additions done by the CTA tier
    CNT_FAST_INLINE, // CTA-tier short-addend additions whose addend was an inline apparent column
    CNT_FAST_SLOT,   // ... whose addend was read through the pivot entry and the arena
    CNT_NUM
};

struct Device {
    int64_t n = 0;        // columns
    int64_t nnz = 0;
    int64_t cap_n = 0;    // allocated column capacity
    int64_t cap_nnz = 0;
    // input in filtration order
    int32_t* in_dims = nullptr;
    int64_t* in_colptr = nullptr;
    int32_t* in_rows = nullptr;
    // reordered matrix
    int32_t* dim = nullptr;      // reordered dims
    int32_t* perm = nullptr;     // reordered -> input
    int32_t* newidx = nullptr;   // input -> reordered
    int64_t* scratch64 = nullptr;   // n+1 int64 (scans)
    // arena of columns
    int32_t* arena = nullptr;
    int64_t arena_cap = 0;       // ints
    unsigned long long* arena_top = nullptr;
    uint64_t* desc = nullptr;
    int32_t* low = nullptr;
    uint64_t* pivot = nullptr;   // [n] pivot entries (see pv_pack)
    uint8_t* state = nullptr;
    uint8_t* cleared = nullptr;
    uint8_t* negative = nullptr;
    int32_t* leftmost = nullptr;
    int32_t* active = nullptr;
    int32_t* runlist = nullptr;  // [n] a step's runnable columns (warp tier input)
    // block-scan scratch
    int64_t* blk = nullptr;      // block sums
    int64_t cap_blk = 0;
    int32_t* dimcnt = nullptr;   // [nblocks * kNumDims]
    int64_t cap_dimcnt = 0;
    DimInfo* diminfo = nullptr;
    unsigned long long* dimtot = nullptr;  // [kNumDims] input columns per dimension (validation pass)
    int* err = nullptr;
    long long* counters = nullptr;
    int* step_ctr = nullptr;     // per-step work counters (8 ints per step)
    int32_t* heavy = nullptr;    // pool of columns handed to the CTA tier, appended step after step
    int64_t pool_cap = 0;
    int* pool_tail = nullptr;
    int* heavy_done = nullptr;   // pool columns the CTA tier has finished (this run)
    int* gate_host = nullptr;    // device view of a mapped host word that mirrors heavy_done
                                 // (owned by the context; null: no mirror)
    int64_t cap_steps = 0;
    // pairs output (input indices)
    int64_t* death_of = nullptr;   // [n]
    int64_t* pairs = nullptr;      // [2n]
    int64_t* ess = nullptr;        // [n]
    int64_t* misc = nullptr;       // [8] small device scalars of the dualization
    // [n] per row owned by an apparent pair whose column holds at most 4
    // entries: {entries below the top, then up to 3 of them}; x = -1 otherwise.
    // Apparent owners never change, so the reduction reads an addend here with
    // one load that does not wait for the pivot entry.
    int4* app = nullptr;
};

}  // namespace sspp
