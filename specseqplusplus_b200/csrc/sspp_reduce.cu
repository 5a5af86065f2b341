// The reduction: lock-free pivot claiming with warp-level sorted-set XOR merges.
//
// Reference counterparts:
//   spectral-sequence block loop       include/specseq.h:592-704 (GPU_Compute)
//   pivot claim + addition queue       include/kernel.h:583-633 (BlockScan, BlockGenAddition)
//   column addition, warp / block      include/kernel.h:691-936, 939-1065
//                                      (cal_rank_*, arr_compact_*, ProcColumnPair*)
//   CPU tail stage                     include/specseq.h:705-1046 (no counterpart here:
//                                      every column is finished on the device)
//
// Design.  One warp reduces one column at a time.  The working column lives in
// shared memory (capacity = level-1 capacity); each addition stages the pivot
// column into shared memory with 16-byte vector loads, merges the two sorted
// index lists (symmetric difference, equal indices cancel) by rank: every
// element's output slot is its own index plus its rank in the other list minus
// twice the cancelled pairs before it (warp ballot + popcount), so no atomics
// and no scratch in global memory.  A column that outgrows shared memory
// continues in global memory (arena buffers of exact size).
//
// Pivot table.  pivot[row] holds the column that owns the row (-1 = none).  A
// column whose lowest row L has no owner, or an owner with a larger index,
// publishes its current entries (fresh arena space, then its descriptor) and
// claims L with a compare-and-swap.  Published column versions are never
// modified afterwards, so a reader holding an older version still adds a valid
// earlier column with the same lowest row.  Displacing a larger owner hands that
// owner to the displacing warp, which reduces it next (it is the only warp
// that can reach it), so no work queue and no spin-wait is needed.  Every
// addition adds an earlier column with the same lowest row, so the result is a
// left-to-right reduction and the pairs equal those of any sequential one.
// Claiming a row also clears the row's own column (twist clearing).
#include <climits>

#include "sspp_kernels.cuh"
#include "sspp_launch.h"

namespace sspp {

struct ReduceArgs {
    const int32_t* active;
    int32_t beg, end;
    int32_t minrow;
    int32_t cap;          // shared-memory capacity per buffer (ints), multiple of 32
    int32_t* arena;
    int64_t arena_cap;
    unsigned long long* arena_top;
    uint64_t* desc;
    int32_t* low;
    int32_t* pivot;
    uint8_t* state;
    uint8_t* cleared;
    int* chunk_ctr;
    int* err;
    long long* counters;
};

constexpr int kMaxMergesPerColumn = 1 << 24;

__device__ __forceinline__ int ldv(const int32_t* p, bool global) { return global ? __ldcg(p) : *p; }

// first index k in [0, n) with a[k] >= x
__device__ __forceinline__ int lower_bound_v(const int32_t* a, int n, int x, bool g) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (ldv(a + mid, g) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// number of indices common to sorted lists a and b
__device__ int warp_count_common(const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb) {
    const int lane = lane_id();
    int e = 0;
    // search the shorter list's elements in the longer list
    if (na > nb) {
        const int32_t* t = a; a = b; b = t;
        int tn = na; na = nb; nb = tn;
        bool tg = ga; ga = gb; gb = tg;
    }
    for (int i = lane; i < na; i += 32) {
        int x = ldv(a + i, ga);
        int r = lower_bound_v(b, nb, x, gb);
        e += (r < nb && ldv(b + r, gb) == x);
    }
    return warp_sum(e);
}

// scatter the survivors of `a` (those not in b) to out at i + rank_b - 2 * cancelled_before
__device__ void warp_scatter_side(const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb, int32_t* out,
                                  int out_len, int* err) {
    const int lane = lane_id();
    int carry = 0;
    for (int base = 0; base < na; base += 32) {
        int i = base + lane;
        bool valid = i < na;
        int x = valid ? ldv(a + i, ga) : 0;
        int r = valid ? lower_bound_v(b, nb, x, gb) : 0;
        bool eq = valid && r < nb && ldv(b + r, gb) == x;
        unsigned m = __ballot_sync(kFull, eq);
        int before = carry + __popc(m & lanemask_lt());
        int pos = i + r - 2 * before;
        if (valid && !eq) {
            if (pos >= 0 && pos < out_len) out[pos] = x;
            else atomicOr(err, ERRB_BAD_INPUT);  // inputs were not strictly increasing
        }
        carry += __popc(m);
    }
}

// out = a xor b (as index sets); out_len known in advance
__device__ __forceinline__ void warp_xor_merge(const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb,
                                               int32_t* out, int out_len, int* err) {
    warp_scatter_side(a, na, ga, b, nb, gb, out, out_len, err);
    warp_scatter_side(b, nb, gb, a, na, ga, out, out_len, err);
    // pad to a multiple of four with INT_MAX (keeps 16-byte vector loads in bounds)
    const int lane = lane_id();
    if (lane < int(pad4(out_len) - out_len)) out[out_len + lane] = INT_MAX;
    __syncwarp();
}

// global -> shared copy of a padded column (16-byte aligned on both sides)
__device__ __forceinline__ void warp_stage(int32_t* dst, const int32_t* src, int len) {
    const int lane = lane_id();
    const int n4 = int(pad4(len)) >> 2;
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = lane; k < n4; k += 32) d4[k] = __ldcg(s4 + k);
    __syncwarp();
}

// shared -> global copy (destination padded to a multiple of four)
__device__ __forceinline__ void warp_store(int32_t* dst, const int32_t* src, int len) {
    const int lane = lane_id();
    const int n4 = int(pad4(len)) >> 2;
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = lane; k < n4; k += 32) d4[k] = s4[k];
}

// Bump allocation of `ints` (multiple of 4) in the arena; -1 when exhausted.
__device__ __forceinline__ int64_t warp_alloc(const ReduceArgs& A, int64_t ints) {
    unsigned long long off = 0;
    if (lane_id() == 0) {
        off = atomicAdd(A.arena_top, (unsigned long long)ints);
        if (int64_t(off) + ints > A.arena_cap) {
            atomicOr(A.err, ERRB_CAPACITY);
            off = ~0ull;
        }
    }
    off = __shfl_sync(kFull, off, 0);
    return off == ~0ull ? -1 : int64_t(off);
}

// Working column of one warp.
struct Work {
    int32_t* buf;      // current entries (shared or arena)
    int len;
    bool global;       // buf is an arena buffer
    int64_t goff;      // arena offset of buf when global
    bool dirty;        // differs from the published version
};

// Makes the working column the published version of `col`.  Returns false
// when the arena is exhausted.
__device__ bool publish(const ReduceArgs& A, int col, Work& w) {
    const int lane = lane_id();
    int64_t off;
    if (w.global) {
        off = w.goff;
    } else {
        off = warp_alloc(A, pad4(w.len));
        if (off < 0) return false;
        warp_store(A.arena + off, w.buf, w.len);
        if (lane == 0) cnt_add(&A.counters[CNT_PUBLISHED], (long long)pad4(w.len));
    }
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        A.desc[col] = pack_desc(uint64_t(off), uint32_t(w.len));
    }
    __syncwarp();
    w.dirty = false;
    return true;
}

enum Outcome { OUT_OWNER, OUT_ZERO, OUT_PARKED, OUT_FAIL };

// Reduces column `col` until it owns its lowest row, becomes zero, or its
// lowest row drops below the band.  *displaced receives the owner this column
// displaced (or -1).
__device__ Outcome reduce_column(const ReduceArgs& A, int col, int32_t* sw0, int32_t* sw1, int32_t* sp,
                                 int* displaced) {
    const int lane = lane_id();
    *displaced = -1;
    uint64_t d = 0;
    if (lane == 0) d = ld_cg_u64(A.desc + col);
    d = __shfl_sync(kFull, d, 0);
    Work w;
    w.len = int(desc_len(d));
    w.dirty = false;
    if (w.len <= A.cap) {
        warp_stage(sw0, A.arena + desc_off(d), w.len);
        w.buf = sw0;
        w.global = false;
        w.goff = 0;
    } else {
        w.buf = A.arena + desc_off(d);
        w.global = true;
        w.goff = int64_t(desc_off(d));
    }
    long long adds = 0, add_ints = 0;
    Outcome res = OUT_FAIL;
    for (int iter = 0;; iter++) {
        if (w.len == 0) {
            if (lane == 0) {
                A.desc[col] = pack_desc(0, 0);
                A.low[col] = -1;
            }
            res = OUT_ZERO;
            break;
        }
        if (iter > kMaxMergesPerColumn) {
            if (lane == 0) atomicOr(A.err, ERRB_TIMEOUT);
            break;
        }
        const int L = ldv(w.buf + w.len - 1, w.global);
        if (L < A.minrow) {
            if (w.dirty && !publish(A, col, w)) break;
            if (lane == 0) A.low[col] = L;
            res = OUT_PARKED;
            break;
        }
        int p = 0;
        if (lane == 0) p = ld_acquire(A.pivot + L);
        p = __shfl_sync(kFull, p, 0);
        if (p < 0 || p > col) {
            if (w.dirty && !publish(A, col, w)) break;
            int old = 0;
            if (lane == 0) {
                A.low[col] = L;
                __threadfence();
                old = atomicCAS(A.pivot + L, p, col);
            }
            old = __shfl_sync(kFull, old, 0);
            if (old == p) {
                if (lane == 0) {
                    if (p < 0) A.cleared[L] = 1;  // twist clearing of the positive row column
                    else cnt_add(&A.counters[CNT_DISPLACED], 1ll);
                }
                *displaced = p;
                res = OUT_OWNER;
                break;
            }
            continue;  // someone else changed the owner; look again
        }
        // add column p (p < col, same lowest row)
        __syncwarp();
        uint64_t dp = 0;
        if (lane == 0) dp = ld_cg_u64(A.desc + p);
        dp = __shfl_sync(kFull, dp, 0);
        const int plen = int(desc_len(dp));
        const int32_t* pb;
        bool pg;
        if (plen <= A.cap) {
            warp_stage(sp, A.arena + desc_off(dp), plen);
            pb = sp;
            pg = false;
        } else {
            pb = A.arena + desc_off(dp);
            pg = true;
        }
        const int common = warp_count_common(w.buf, w.len, w.global, pb, plen, pg);
        const int out_len = w.len + plen - 2 * common;
        if (out_len > int(kMaxColLen)) {
            if (lane == 0) atomicOr(A.err, ERRB_LEN);
            break;
        }
        adds++;
        add_ints += w.len + plen + out_len;
        if (out_len <= A.cap) {
            int32_t* dst = (w.global || w.buf == sw1) ? sw0 : sw1;
            warp_xor_merge(w.buf, w.len, w.global, pb, plen, pg, dst, out_len, A.err);
            w.buf = dst;
            w.global = false;
        } else {
            int64_t off = warp_alloc(A, pad4(out_len));
            if (off < 0) break;
            warp_xor_merge(w.buf, w.len, w.global, pb, plen, pg, A.arena + off, out_len, A.err);
            __syncwarp();
            if (lane == 0) cnt_add(&A.counters[CNT_PUBLISHED], (long long)pad4(out_len));
            w.buf = A.arena + off;
            w.global = true;
            w.goff = off;
        }
        w.len = out_len;
        w.dirty = true;
    }
    if (lane == 0 && adds) {
        cnt_add(&A.counters[CNT_ADDITIONS], adds);
        cnt_add(&A.counters[CNT_ADD_INTS], add_ints);
    }
    return res;
}

__global__ void __launch_bounds__(128) k_reduce_step(ReduceArgs A) {
    extern __shared__ __align__(16) int32_t smem[];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    int32_t* sw0 = smem + size_t(wib) * 3 * A.cap;
    int32_t* sw1 = sw0 + A.cap;
    int32_t* sp = sw1 + A.cap;
    const int count = A.end - A.beg;
    while (true) {
        int base = 0;
        if (lane == 0) base = atomicAdd(A.chunk_ctr, 32);
        base = __shfl_sync(kFull, base, 0);
        if (base >= count) break;
        const int idx = A.beg + base + lane;
        int c = -1;
        bool run = false;
        if (idx < A.end) {
            c = A.active[idx];
            run = ld_acquire_u8(A.state + c) == ST_ACTIVE && !ld_acquire_u8(A.cleared + c) &&
                  __ldcg(A.low + c) >= A.minrow;
        }
        unsigned m = __ballot_sync(kFull, run);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            int col = __shfl_sync(kFull, c, src);
            // the column and any owners it displaces, one after another
            while (col >= 0) {
                int next = -1;
                Outcome o = reduce_column(A, col, sw0, sw1, sp, &next);
                if (lane == 0) {
                    if (o == OUT_OWNER) A.state[col] = ST_OWNER;
                    else if (o == OUT_ZERO) A.state[col] = ST_ZERO;
                    else if (o == OUT_PARKED) { __threadfence(); st_release_u8(A.state + col, ST_ACTIVE); }
                    else st_release_u8(A.state + col, ST_ACTIVE);  // failure: left for a retry
                }
                __syncwarp();
                if (o == OUT_FAIL) return;
                col = next;
            }
        }
    }
}

int reduce_smem_bytes(int cap) { return 4 * 3 * cap * 4; }

void reduce_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                   int* chunk_ctr, int grid, cudaStream_t s) {
    ReduceArgs A;
    A.active = active;
    A.beg = beg;
    A.end = end;
    A.minrow = minrow;
    A.cap = cap;
    A.arena = D.arena;
    A.arena_cap = D.arena_cap;
    A.arena_top = D.arena_top;
    A.desc = D.desc;
    A.low = D.low;
    A.pivot = D.pivot;
    A.state = D.state;
    A.cleared = D.cleared;
    A.chunk_ctr = chunk_ctr;
    A.err = D.err;
    A.counters = D.counters;
    k_reduce_step<<<grid, 128, reduce_smem_bytes(cap), s>>>(A);
}

cudaError_t reduce_configure(int cap, int* blocks_per_sm) {
    int bytes = reduce_smem_bytes(cap);
    cudaError_t e = cudaFuncSetAttribute(k_reduce_step, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_reduce_step, 128, bytes);
}

}  // namespace sspp
