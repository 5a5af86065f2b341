// The reduction: lock-free pivot claiming with group-parallel sorted-set XOR merges.
//
// Reference counterparts:
//   spectral-sequence block loop       include/specseq.h:592-704 (GPU_Compute)
//   pivot claim + addition queue       include/kernel.h:583-633 (BlockScan, BlockGenAddition)
//   column addition, warp phase        include/kernel.h:691-743, 814-936 (ProcColumnPair)
//   column addition, block phase       include/kernel.h:744-792, 939-1065 (ProcColumnPair_121Block)
//   CPU tail stage                     include/specseq.h:705-1046 (no counterpart here:
//                                      every column is finished on the device)
//
// Two tiers, as in the reference's two phases.  Light tier: one warp reduces
// one column whose entries fit in the warp's shared-memory buffers (level-1
// capacity).  Heavy tier: a column that outgrows them is handed to a second
// kernel in which a whole CTA reduces it with buffers of the level-2 capacity,
// and beyond that in exact-size arena buffers.  Both tiers run the same
// column routine, written once over a "group" (warp or CTA).
//
// Merge.  Each addition stages the pivot column into shared memory with
// 16-byte vector loads and merges the two sorted index lists (symmetric
// difference: equal indices cancel) by rank: an element's output slot is its
// own index plus its rank in the other list minus twice the cancelled pairs
// before it (ballot + popcount prefix), so no atomics and no global scratch.
//
// Pivot table.  pivot[row] holds the column that owns the row (-1 = none).  A
// column whose lowest row L has no owner, or an owner with a larger index,
// publishes its current entries (fresh arena space, then its descriptor) and
// claims L with a compare-and-swap.  Published column versions are never
// modified afterwards, so a reader holding an older version still adds a valid
// earlier column with the same lowest row.  Displacing a larger owner hands that
// owner to the displacing group, which reduces it next (no other group can
// reach it), so there is no work queue to wait on and no spin-wait at all.
// Every addition adds an earlier column with the same lowest row, so the
// result is a left-to-right reduction and the pairs equal those of any
// sequential one.  Claiming a row also clears the row's own column (twist).
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
    int* ctr;             // [0] chunk counter, [1] heavy list length, [2] heavy pull counter
    int32_t* heavy;       // heavy list
    int* err;
    long long* counters;
};

constexpr int kMaxMergesPerColumn = 1 << 24;

// ------------------------------------------------------------------ groups
struct WarpG {
    static constexpr int kSize = 32;
    __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
    __device__ __forceinline__ bool leader() const { return (threadIdx.x & 31) == 0; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ int bcast(int v) const { return __shfl_sync(kFull, v, 0); }
    __device__ __forceinline__ unsigned long long bcast64(unsigned long long v) const {
        return __shfl_sync(kFull, v, 0);
    }
    // exclusive count of f over lower ranks; tot = count over the group
    __device__ __forceinline__ int prefix(bool f, int& tot) const {
        unsigned m = __ballot_sync(kFull, f);
        tot = __popc(m);
        return __popc(m & lanemask_lt());
    }
    __device__ __forceinline__ int sum(int v) const { return warp_sum(v); }
};

template <int T>
struct BlockG {
    static constexpr int kSize = T;
    static constexpr int kWarps = T / 32;
    int* sm;                  // kWarps + 2 ints
    unsigned long long* sb;   // one 8-byte slot
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ unsigned long long bcast64(unsigned long long v) const {
        if (threadIdx.x == 0) *sb = v;
        __syncthreads();
        unsigned long long r = *sb;
        __syncthreads();
        return r;
    }
    __device__ __forceinline__ int bcast(int v) const { return int(bcast64((unsigned long long)(unsigned)v)); }
    __device__ __forceinline__ int prefix(bool f, int& tot) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        unsigned m = __ballot_sync(kFull, f);
        if (lane == 0) sm[wid] = __popc(m);
        __syncthreads();
        if (wid == 0) {
            int c = lane < kWarps ? sm[lane] : 0;
            int inc = warp_inclusive_scan(c);
            if (lane < kWarps) sm[lane] = inc - c;
            if (lane == kWarps - 1) sm[kWarps] = inc;
        }
        __syncthreads();
        int r = sm[wid] + __popc(m & lanemask_lt());
        tot = sm[kWarps];
        __syncthreads();
        return r;
    }
    __device__ __forceinline__ int sum(int v) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int w = warp_sum(v);
        if (lane == 0) sm[wid] = w;
        __syncthreads();
        if (wid == 0) {
            int c = lane < kWarps ? sm[lane] : 0;
            c = warp_sum(c);
            if (lane == 0) sm[kWarps] = c;
        }
        __syncthreads();
        int r = sm[kWarps];
        __syncthreads();
        return r;
    }
};

// --------------------------------------------------------------- list ops
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
template <class G>
__device__ int count_common(const G& g, const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb) {
    if (na > nb) {  // search the shorter list's elements in the longer one
        const int32_t* t = a; a = b; b = t;
        int tn = na; na = nb; nb = tn;
        bool tg = ga; ga = gb; gb = tg;
    }
    int e = 0;
    for (int i = g.rank(); i < na; i += G::kSize) {
        int x = ldv(a + i, ga);
        int r = lower_bound_v(b, nb, x, gb);
        e += (r < nb && ldv(b + r, gb) == x);
    }
    return g.sum(e);
}

// survivors of a (those not in b) go to out[i + rank_b(x) - 2 * cancelled_before(i)]
template <class G>
__device__ void scatter_side(const G& g, const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb,
                             int32_t* out, int out_len, int* err) {
    int carry = 0;
    for (int base = 0; base < na; base += G::kSize) {
        int i = base + g.rank();
        bool valid = i < na;
        int x = valid ? ldv(a + i, ga) : 0;
        int r = valid ? lower_bound_v(b, nb, x, gb) : 0;
        bool eq = valid && r < nb && ldv(b + r, gb) == x;
        int tot;
        int before = carry + g.prefix(eq, tot);
        if (valid && !eq) {
            int pos = i + r - 2 * before;
            if (pos >= 0 && pos < out_len) out[pos] = x;
            else atomicOr(err, ERRB_BAD_INPUT);  // inputs were not strictly increasing
        }
        carry += tot;
    }
}

template <class G>
__device__ void xor_merge(const G& g, const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb,
                          int32_t* out, int out_len, int* err) {
    scatter_side(g, a, na, ga, b, nb, gb, out, out_len, err);
    scatter_side(g, b, nb, gb, a, na, ga, out, out_len, err);
    // pad to a multiple of four with INT_MAX (keeps 16-byte vector loads in bounds)
    if (g.rank() < int(pad4(out_len) - out_len)) out[out_len + g.rank()] = INT_MAX;
    g.sync();
}

// global -> shared copy of a padded column (16-byte aligned on both sides)
template <class G>
__device__ __forceinline__ void stage(const G& g, int32_t* dst, const int32_t* src, int len) {
    const int n4 = int(pad4(len)) >> 2;
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = g.rank(); k < n4; k += G::kSize) d4[k] = __ldcg(s4 + k);
    g.sync();
}

template <class G>
__device__ __forceinline__ void store(const G& g, int32_t* dst, const int32_t* src, int len) {
    const int n4 = int(pad4(len)) >> 2;
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = g.rank(); k < n4; k += G::kSize) d4[k] = s4[k];
}

// Bump allocation of `ints` (multiple of 4) in the arena; -1 when exhausted.
template <class G>
__device__ __forceinline__ int64_t alloc(const G& g, const ReduceArgs& A, int64_t ints) {
    unsigned long long off = 0;
    if (g.leader()) {
        off = atomicAdd(A.arena_top, (unsigned long long)ints);
        if (int64_t(off) + ints > A.arena_cap) {
            atomicOr(A.err, ERRB_CAPACITY);
            off = ~0ull;
        }
    }
    off = g.bcast64(off);
    return off == ~0ull ? -1 : int64_t(off);
}

// Working column of one group.
struct Work {
    int32_t* buf;      // current entries (shared or arena)
    int len;
    bool global;       // buf is an arena buffer
    int64_t goff;      // arena offset of buf when global
    bool dirty;        // differs from the published version
};

// Makes the working column the published version of `col`; false when the
// arena is exhausted.
template <class G>
__device__ bool publish(const G& g, const ReduceArgs& A, int col, Work& w) {
    int64_t off;
    if (w.global) {
        off = w.goff;
    } else {
        off = alloc(g, A, pad4(w.len));
        if (off < 0) return false;
        store(g, A.arena + off, w.buf, w.len);
        if (g.leader()) cnt_add(&A.counters[CNT_PUBLISHED], (long long)pad4(w.len));
    }
    g.sync();
    if (g.leader()) {
        __threadfence();
        A.desc[col] = pack_desc(uint64_t(off), uint32_t(w.len));
    }
    g.sync();
    w.dirty = false;
    return true;
}

enum Outcome { OUT_OWNER, OUT_ZERO, OUT_PARKED, OUT_DEFERRED, OUT_FAIL };

// Reduces column `col` until it owns its lowest row, becomes zero, or its
// lowest row drops below the band.  With `defer`, a column whose entries (or
// whose next addend or sum) exceed the shared capacity is published and
// returned as OUT_DEFERRED for the heavy tier; without it such columns continue
// in arena buffers.  *displaced receives the owner this column displaced (-1
// if none).
template <class G>
__device__ Outcome reduce_column(const G& g, const ReduceArgs& A, int col, int32_t* sw0, int32_t* sw1, int32_t* sp,
                                 bool defer, int* displaced) {
    *displaced = -1;
    uint64_t d = 0;
    if (g.leader()) d = ld_cg_u64(A.desc + col);
    d = g.bcast64(d);
    Work w;
    w.len = int(desc_len(d));
    w.dirty = false;
    if (w.len <= A.cap) {
        stage(g, sw0, A.arena + desc_off(d), w.len);
        w.buf = sw0;
        w.global = false;
        w.goff = 0;
    } else if (defer) {
        return OUT_DEFERRED;
    } else {
        w.buf = A.arena + desc_off(d);
        w.global = true;
        w.goff = int64_t(desc_off(d));
    }
    long long adds = 0, add_ints = 0;
    Outcome res = OUT_FAIL;
    for (int iter = 0;; iter++) {
        if (w.len == 0) {
            if (g.leader()) {
                A.desc[col] = pack_desc(0, 0);
                A.low[col] = -1;
            }
            res = OUT_ZERO;
            break;
        }
        if (iter > kMaxMergesPerColumn) {
            if (g.leader()) atomicOr(A.err, ERRB_TIMEOUT);
            break;
        }
        const int L = ldv(w.buf + w.len - 1, w.global);
        if (L < A.minrow) {
            if (w.dirty && !publish(g, A, col, w)) break;
            if (g.leader()) A.low[col] = L;
            res = OUT_PARKED;
            break;
        }
        int p = 0;
        if (g.leader()) p = ld_acquire(A.pivot + L);
        p = g.bcast(p);
        if (p < 0 || p > col) {
            if (w.dirty && !publish(g, A, col, w)) break;
            int old = 0;
            if (g.leader()) {
                A.low[col] = L;
                __threadfence();
                old = atomicCAS(A.pivot + L, p, col);
            }
            old = g.bcast(old);
            if (old == p) {
                if (g.leader()) {
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
        g.sync();
        uint64_t dp = 0;
        if (g.leader()) dp = ld_cg_u64(A.desc + p);
        dp = g.bcast64(dp);
        const int plen = int(desc_len(dp));
        const int32_t* pb;
        bool pg;
        if (plen <= A.cap) {
            stage(g, sp, A.arena + desc_off(dp), plen);
            pb = sp;
            pg = false;
        } else if (defer) {
            if (w.dirty && !publish(g, A, col, w)) break;
            res = OUT_DEFERRED;
            break;
        } else {
            pb = A.arena + desc_off(dp);
            pg = true;
        }
        const int common = count_common(g, w.buf, w.len, w.global, pb, plen, pg);
        const int out_len = w.len + plen - 2 * common;
        if (out_len > int(kMaxColLen)) {
            if (g.leader()) atomicOr(A.err, ERRB_LEN);
            break;
        }
        if (out_len > A.cap && defer) {
            if (w.dirty && !publish(g, A, col, w)) break;
            res = OUT_DEFERRED;
            break;
        }
        adds++;
        add_ints += w.len + plen + out_len;
        if (out_len <= A.cap) {
            int32_t* dst = (w.global || w.buf == sw1) ? sw0 : sw1;
            xor_merge(g, w.buf, w.len, w.global, pb, plen, pg, dst, out_len, A.err);
            w.buf = dst;
            w.global = false;
        } else {
            int64_t off = alloc(g, A, pad4(out_len));
            if (off < 0) break;
            xor_merge(g, w.buf, w.len, w.global, pb, plen, pg, A.arena + off, out_len, A.err);
            if (g.leader()) cnt_add(&A.counters[CNT_PUBLISHED], (long long)pad4(out_len));
            w.buf = A.arena + off;
            w.global = true;
            w.goff = off;
        }
        w.len = out_len;
        w.dirty = true;
    }
    if (g.leader() && adds) {
        cnt_add(&A.counters[CNT_ADDITIONS], adds);
        cnt_add(&A.counters[CNT_ADD_INTS], add_ints);
    }
    return res;
}

// Final state of a column after reduce_column; returns false on failure.
template <class G>
__device__ __forceinline__ bool settle(const G& g, const ReduceArgs& A, int col, Outcome o) {
    if (g.leader()) {
        switch (o) {
            case OUT_OWNER: A.state[col] = ST_OWNER; break;
            case OUT_ZERO: A.state[col] = ST_ZERO; break;
            case OUT_DEFERRED:
                A.state[col] = ST_HEAVY;
                A.heavy[atomicAdd(A.ctr + 1, 1)] = col;
                break;
            default: __threadfence(); st_release_u8(A.state + col, ST_ACTIVE); break;  // parked / failed
        }
    }
    g.sync();
    return o != OUT_FAIL;
}

// Light tier: warps take chunks of 32 window entries and reduce the runnable
// ones (active, not cleared, lowest row inside the band) one after another.
__global__ void __launch_bounds__(128) k_reduce_light(ReduceArgs A) {
    extern __shared__ __align__(16) int32_t smem[];
    WarpG g;
    const int lane = g.rank();
    int32_t* sw0 = smem + size_t(threadIdx.x >> 5) * 3 * A.cap;
    int32_t* sw1 = sw0 + A.cap;
    int32_t* sp = sw1 + A.cap;
    const int count = A.end - A.beg;
    while (true) {
        int base = 0;
        if (lane == 0) base = atomicAdd(A.ctr, 32);
        base = g.bcast(base);
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
            while (col >= 0) {  // the column, then any owner it displaced
                int next = -1;
                Outcome o = reduce_column(g, A, col, sw0, sw1, sp, true, &next);
                if (!settle(g, A, col, o)) return;
                col = next;
            }
        }
    }
}

// Heavy tier: one CTA per deferred column, buffers of the level-2 capacity.
template <int T>
__global__ void __launch_bounds__(T) k_reduce_heavy(ReduceArgs A) {
    extern __shared__ __align__(16) int32_t smem[];
    __shared__ int gsm[T / 32 + 2];
    __shared__ unsigned long long gsb;
    BlockG<T> g;
    g.sm = gsm;
    g.sb = &gsb;
    int32_t* sw0 = smem;
    int32_t* sw1 = sw0 + A.cap;
    int32_t* sp = sw1 + A.cap;
    const int nheavy = __ldcg(A.ctr + 1);
    while (true) {
        int k = 0;
        if (g.leader()) k = atomicAdd(A.ctr + 2, 1);
        k = g.bcast(k);
        if (k >= nheavy) break;
        int col = __ldcg(A.heavy + k);
        while (col >= 0) {
            int next = -1;
            Outcome o = reduce_column(g, A, col, sw0, sw1, sp, false, &next);
            if (!settle(g, A, col, o)) return;
            col = next;
        }
    }
}

constexpr int kHeavyThreads = 256;

int light_smem_bytes(int cap) { return 4 * 3 * cap * 4; }
int heavy_smem_bytes(int cap) { return 3 * cap * 4; }

static ReduceArgs make_args(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                            int* ctr) {
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
    A.ctr = ctr;
    A.heavy = D.heavy;
    A.err = D.err;
    A.counters = D.counters;
    return A;
}

void reduce_light_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                         int* ctr, int grid, cudaStream_t s) {
    k_reduce_light<<<grid, 128, light_smem_bytes(cap), s>>>(make_args(D, active, beg, end, minrow, cap, ctr));
}

void reduce_heavy_launch(const Device& D, int32_t minrow, int cap, int* ctr, int grid, cudaStream_t s) {
    k_reduce_heavy<kHeavyThreads><<<grid, kHeavyThreads, heavy_smem_bytes(cap), s>>>(
        make_args(D, nullptr, 0, 0, minrow, cap, ctr));
}

cudaError_t reduce_configure(int cap1, int cap2, int* light_blocks_per_sm, int* heavy_blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(k_reduce_light, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         light_smem_bytes(cap1));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(light_blocks_per_sm, k_reduce_light, 128, light_smem_bytes(cap1));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_reduce_heavy<kHeavyThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             heavy_smem_bytes(cap2));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(heavy_blocks_per_sm, k_reduce_heavy<kHeavyThreads>,
                                                         kHeavyThreads, heavy_smem_bytes(cap2));
}

}  // namespace sspp
