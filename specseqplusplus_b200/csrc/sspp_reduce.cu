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
// Pivot table.  pivot[row] holds the owning column and the arena slot of the
// owner's version (pv_pack), so the owner's entries are one dependent load
// away.  A column whose lowest row L has no owner, or an owner with a larger
// index, publishes its current entries (fresh arena slot, then its
// descriptor) and claims L with a 64-bit compare-and-swap.  Published column
// versions are never modified afterwards, so a reader holding an older entry
// still adds a valid earlier column with the same lowest row.  Displacing a
// larger owner hands that owner to the displacing group, which reduces it
// next (no other group can reach it), so there is no work queue to wait on and
// no spin-wait at all.  Every addition adds an earlier column with the same
// lowest row, so the result is a left-to-right reduction and the pairs equal
// those of any sequential one.  Claiming a row also clears the row's own
// column (twist clearing).
//
// Addition.  The addend is staged into shared memory with 16-byte vector loads
// (header and entries in one round when it fits).  The next lowest row is
// known before the merge - it is the largest index at which the tops of the
// two lists stop agreeing - so the pivot entry of that row is requested before
// the merge starts and arrives while it runs.  The merge computes each
// element's output slot from its rank in the other list minus twice the
// cancelled pairs before it (one ballot/prefix per round for both lists): no
// atomics, no scratch in global memory.
#include <climits>
#include <mutex>

#include "sspp_kernels.cuh"
#include "sspp_launch.h"

namespace sspp {

struct ReduceArgs {
    int32_t ncols;
    const int32_t* active;
    int32_t beg, end;
    int32_t minrow;
    int32_t cap;          // shared-memory capacity per buffer (ints), multiple of 32
    int32_t chunk;        // light tier: window entries taken per fetch (1..32)
    int32_t* arena;
    int64_t arena_cap;
    unsigned long long* arena_top;
    uint64_t* desc;
    int32_t* low;
    uint64_t* pivot;
    uint8_t* state;
    uint8_t* cleared;
    int* ctr;             // per step: [0] chunk counter, [1] [2] heavy pool range, [3] heavy pull counter,
                          // [4] warp-tier blocks finished, [5] runnable columns listed by k_light_filter
    const int* count;     // when set, the work is active[beg, beg + *count) (a filtered list)
    int* ctr_next;        // the next step's counters (its pool range starts where this step's ends), or null
    int32_t* heavy;       // heavy pool (columns handed to the CTA tier, appended in step order)
    int* pool_tail;
    int* heavy_done;      // pool columns finished by the CTA tier
    int* gate_host;       // mapped host mirror of heavy_done, or null
    int64_t pool_cap;
    int* err;
    long long* counters;
    int32_t light_chain;  // warp tier: additions per column before handing it to the CTA tier (0 = no limit)
    const int4* app;      // inline short apparent columns by row (Device::app)
};

// Where one reduction of a column stops: the band's lowest row (a column whose
// low drops below it parks), and the counter of the work it came from, so that
// a long chain in the warp tier moves to the CTA tier once that work is fully
// handed out (drain_ctr >= drain_total).
struct Band {
    int32_t minrow;
    const int* drain_ctr;
    int32_t drain_total;
};

constexpr int kMaxMergesPerColumn = 1 << 24;

// A pivot entry read early, before it is known whether it is needed: relaxed,
// so a fence (acquire) must come before the owner's slot is read through it.
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// ------------------------------------------------------------------ groups
struct WarpG {
    static constexpr int kSize = 32;
    __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
    __device__ __forceinline__ bool leader() const { return (threadIdx.x & 31) == 0; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    // __syncwarp orders the leader's preceding memory accesses (an acquire in
    // particular) before the other lanes' following ones
    __device__ __forceinline__ int bcast(int v) const {
        __syncwarp();
        return __shfl_sync(kFull, v, 0);
    }
    __device__ __forceinline__ unsigned long long bcast64(unsigned long long v) const {
        __syncwarp();
        return __shfl_sync(kFull, v, 0);
    }
    __device__ __forceinline__ unsigned long long bcast64_last(unsigned long long v) const {
        __syncwarp();
        return __shfl_sync(kFull, v, 31);
    }
    // exclusive counts of fa and fb over lower ranks, and their group totals
    __device__ __forceinline__ void prefix2(bool fa, bool fb, int& pa, int& pb, int& ta, int& tb) const {
        const unsigned lt = lanemask_lt();
        unsigned ma = __ballot_sync(kFull, fa), mb = __ballot_sync(kFull, fb);
        pa = __popc(ma & lt);
        pb = __popc(mb & lt);
        ta = __popc(ma);
        tb = __popc(mb);
    }
    __device__ __forceinline__ int sum(int v) const { return warp_sum(v); }
    // exclusive prefix of v over lower ranks; tot = group total
    __device__ __forceinline__ int prefix_int(int v, int& tot) const {
        int inc = warp_inclusive_scan(v);
        tot = __shfl_sync(kFull, inc, 31);
        return inc - v;
    }
};

template <int T>
struct BlockG {
    static constexpr int kSize = T;
    static constexpr int kWarps = T / 32;
    int* sm;                  // 2 * (kWarps + 2) ints: two scan buffers, used alternately
    unsigned long long* sb;   // two 8-byte broadcast slots, used alternately
    mutable int slot = 0;
    mutable int sbuf = 0;
    // alternating buffers: buffer b is rewritten only two collectives later,
    // after every thread has passed the barrier of the collective in between
    __device__ __forceinline__ int* scan_buf() const {
        int* b = sm + sbuf * (kWarps + 2);
        sbuf ^= 1;
        return b;
    }
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    // one barrier: consecutive broadcasts alternate slots, and a slot is only
    // rewritten after every thread has passed the following broadcast's barrier
    __device__ __forceinline__ unsigned long long bcast64(unsigned long long v) const {
        unsigned long long* p = sb + slot;
        slot ^= 1;
        if (threadIdx.x == 0) *p = v;
        __syncthreads();
        return *p;
    }
    __device__ __forceinline__ int bcast(int v) const { return int(bcast64((unsigned long long)(unsigned)v)); }
    __device__ __forceinline__ unsigned long long bcast64_last(unsigned long long v) const {
        unsigned long long* p = sb + slot;
        slot ^= 1;
        if (threadIdx.x == T - 1) *p = v;
        __syncthreads();
        return *p;
    }
    __device__ __forceinline__ void prefix2(bool fa, bool fb, int& pa, int& pb, int& ta, int& tb) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const unsigned lt = lanemask_lt();
        int* b = scan_buf();
        unsigned ma = __ballot_sync(kFull, fa), mb = __ballot_sync(kFull, fb);
        if (lane == 0) b[wid] = __popc(ma) | (__popc(mb) << 16);
        __syncthreads();
        if (wid == 0) {
            int c = lane < kWarps ? b[lane] : 0;
            int inc = warp_inclusive_scan(c);
            if (lane < kWarps) b[lane] = inc - c;
            if (lane == kWarps - 1) b[kWarps] = inc;
        }
        __syncthreads();
        const int base = b[wid], tot = b[kWarps];
        pa = (base & 0xffff) + __popc(ma & lt);
        pb = (base >> 16) + __popc(mb & lt);
        ta = tot & 0xffff;
        tb = tot >> 16;
    }
    __device__ __forceinline__ int prefix_int(int v, int& tot) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int* b = scan_buf();
        int inc = warp_inclusive_scan(v);
        if (lane == 31) b[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            int c = lane < kWarps ? b[lane] : 0;
            int ci = warp_inclusive_scan(c);
            if (lane < kWarps) b[lane] = ci - c;
            if (lane == kWarps - 1) b[kWarps] = ci;
        }
        __syncthreads();
        tot = b[kWarps];
        return b[wid] + inc - v;
    }
    __device__ __forceinline__ int sum(int v) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int* b = scan_buf();
        int w = warp_sum(v);
        if (lane == 0) b[wid] = w;
        __syncthreads();
        if (wid == 0) {
            int c = lane < kWarps ? b[lane] : 0;
            c = warp_sum(c);
            if (lane == 0) b[kWarps] = c;
        }
        __syncthreads();
        return b[kWarps];
    }
};

// --------------------------------------------------------------- list ops
// List loads: shared-memory lists with ld.shared, arena lists through L2
// (ld.global.cg: arena slots written by other SMs must not be served from a
// stale L1 line).  The space of each list is a template parameter, so no load
// carries a runtime branch or generic addressing.
__device__ __forceinline__ int lds(const int32_t* p) {
    int v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(unsigned(__cvta_generic_to_shared(p))));
    return v;
}
template <bool GL>
__device__ __forceinline__ int ld(const int32_t* p) {
    if constexpr (GL) return __ldcg(p);
    else return lds(p);
}
__device__ __forceinline__ int ldv(const int32_t* p, bool global) { return global ? __ldcg(p) : lds(p); }

// A store the host sees without synchronising (mapped pinned memory); stores
// of different CTAs may land out of order, so the host reads a lower bound.
__device__ __forceinline__ void st_relaxed_sys(int* p, int v) {
    asm volatile("st.relaxed.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// calls F<ga, gb>(...) with the spaces known at compile time
#define SSPP_DISPATCH2(ga, gb, CALL) \
    ((ga) ? ((gb) ? CALL(true, true) : CALL(true, false)) : ((gb) ? CALL(false, true) : CALL(false, false)))

// first index k in [0, n) with a[k] >= x
template <bool GL>
__device__ __forceinline__ int lower_bound_t(const int32_t* a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (ld<GL>(a + mid) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// number of indices common to sorted lists a and b (b is searched)
template <class G, bool GA, bool GB>
__device__ int count_common_t(const G& g, const int32_t* a, int na, const int32_t* b, int nb) {
    int e = 0;
    for (int i = g.rank(); i < na; i += G::kSize) {
        int x = ld<GA>(a + i);
        int r = lower_bound_t<GB>(b, nb, x);
        e += (r < nb && ld<GB>(b + r) == x);
    }
    return g.sum(e);
}

template <class G>
__device__ int count_common(const G& g, const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb) {
    if (na > nb) {  // search the shorter list's elements in the longer one
        const int32_t* t = a; a = b; b = t;
        int tn = na; na = nb; nb = tn;
        bool tg = ga; ga = gb; gb = tg;
    }
#define SSPP_CC(A_, B_) count_common_t<G, A_, B_>(g, a, na, b, nb)
    return SSPP_DISPATCH2(ga, gb, SSPP_CC);
#undef SSPP_CC
}

// out = a xor b (as index sets) in one pass over both lists.  Element a[i]
// survives unless it is in b; it lands at i + rank_b(a[i]) - 2 * (cancelled
// a's before i), symmetrically for b.  Writes stay below out_cap.  Returns the
// output length and pads it to a multiple of four with INT_MAX.
// Two lower-bound searches in lockstep (x in b, y in a): two independent load
// chains per step.  Equality comes from the probe that last moved `hi` (the
// final position was probed then), so no extra dependent load is needed.
template <bool GA, bool GB>
__device__ __forceinline__ void rank2(const int32_t* a, int na, const int32_t* b, int nb, int x, bool vx, int y, bool vy,
                                      int& rx, bool& ex, int& ry, bool& ey) {
    int lo1 = 0, hi1 = vx ? nb : 0, lo2 = 0, hi2 = vy ? na : 0;
    int h1 = INT_MIN, h2 = INT_MIN;
    while (lo1 < hi1 || lo2 < hi2) {
        const bool s1 = lo1 < hi1, s2 = lo2 < hi2;
        const int m1 = (lo1 + hi1) >> 1, m2 = (lo2 + hi2) >> 1;
        const int v1 = s1 ? ld<GB>(b + m1) : 0;
        const int v2 = s2 ? ld<GA>(a + m2) : 0;
        if (s1) {
            if (v1 < x) lo1 = m1 + 1;
            else { hi1 = m1; h1 = v1; }
        }
        if (s2) {
            if (v2 < y) lo2 = m2 + 1;
            else { hi2 = m2; h2 = v2; }
        }
    }
    rx = lo1;
    ex = vx && lo1 < nb && h1 == x;
    ry = lo2;
    ey = vy && lo2 < na && h2 == y;
}

template <class G, bool GA, bool GB>
__device__ int xor_merge(const G& g, const int32_t* a, int na, const int32_t* b, int nb, int32_t* out, int out_cap,
                         int* err) {
    int carry_a = 0, carry_b = 0;
    const int n = na > nb ? na : nb;
    for (int base = 0; base < n; base += G::kSize) {
        const int i = base + g.rank();
        const bool va = i < na, vb = i < nb;
        const int x = va ? ld<GA>(a + i) : 0;
        const int y = vb ? ld<GB>(b + i) : 0;
        int ra, rb;
        bool ea, eb;
        rank2<GA, GB>(a, na, b, nb, x, va, y, vb, ra, ea, rb, eb);
        int pa, pb, ta, tb;
        g.prefix2(ea, eb, pa, pb, ta, tb);
        if (va && !ea) {
            int pos = i + ra - 2 * (carry_a + pa);
            if (pos >= 0 && pos < out_cap) out[pos] = x;
            else atomicOr(err, ERRB_BAD_INPUT);  // inputs were not strictly increasing
        }
        if (vb && !eb) {
            int pos = i + rb - 2 * (carry_b + pb);
            if (pos >= 0 && pos < out_cap) out[pos] = y;
            else atomicOr(err, ERRB_BAD_INPUT);
        }
        carry_a += ta;
        carry_b += tb;
    }
    const int out_len = na + nb - 2 * carry_a;
    const int padn = int(pad4(out_len) - out_len);
    if (g.rank() < padn && out_len + g.rank() < out_cap) out[out_len + g.rank()] = INT_MAX;
    g.sync();
    return out_len;
}

// Merge-path form of the same merge.  M = merge(a, b), a first on ties, so
// every equal pair is adjacent in M as (a[i], b[j]).  Thread t owns positions
// [tK, tK + K) of M per round: one binary search finds its split (i, j), a
// short walk emits the elements of its positions that have no equal partner
// (a pair cut by a slice boundary is dropped on both sides), and a group
// prefix sum of the per-thread counts places them.  The walk runs twice
// (count, then write) so nothing is held in registers.
template <int K, bool GA, bool GB>
__device__ __forceinline__ int path_walk(const int32_t* a, int na, const int32_t* b, int nb, int d0, int total,
                                         int32_t* out, int out_off, int out_cap, bool emit, int* err) {
    int lo = d0 - nb > 0 ? d0 - nb : 0, hi = d0 < na ? d0 : na;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ld<GA>(a + mid - 1) <= ld<GB>(b + d0 - mid)) lo = mid;
        else hi = mid - 1;
    }
    int i = lo, j = d0 - lo, pos = d0, cnt = 0;
    const int end = d0 + K < total ? d0 + K : total;
    // b[j] partners the element just before this slice (a[i-1])
    if (pos < end && i > 0 && j < nb && ld<GA>(a + i - 1) == ld<GB>(b + j)) { j++; pos++; }
    while (pos < end) {
        const int x = i < na ? ld<GA>(a + i) : INT_MAX;
        const int y = j < nb ? ld<GB>(b + j) : INT_MAX;
        if (i < na && (j >= nb || x <= y)) {
            if (j < nb && x == y) {  // equal pair: drop both (the partner may open the next slice)
                i++;
                pos++;
                if (pos < end) { j++; pos++; }
                continue;
            }
            if (emit) {
                if (out_off + cnt < out_cap) out[out_off + cnt] = x;
                else atomicOr(err, ERRB_BAD_INPUT);
            }
            cnt++;
            i++;
        } else {
            if (emit) {
                if (out_off + cnt < out_cap) out[out_off + cnt] = y;
                else atomicOr(err, ERRB_BAD_INPUT);
            }
            cnt++;
            j++;
        }
        pos++;
    }
    return cnt;
}

template <class G, int K, bool GA, bool GB>
__device__ int xor_merge_path(const G& g, const int32_t* a, int na, const int32_t* b, int nb, int32_t* out,
                              int out_cap, int* err) {
    const int total = na + nb;
    int written = 0;
    for (int base = 0; base < total; base += G::kSize * K) {
        const int d0 = base + g.rank() * K;
        int cnt = d0 < total ? path_walk<K, GA, GB>(a, na, b, nb, d0, total, out, 0, out_cap, false, err) : 0;
        int tot;
        const int off = g.prefix_int(cnt, tot);
        if (cnt) path_walk<K, GA, GB>(a, na, b, nb, d0, total, out, written + off, out_cap, true, err);
        written += tot;
    }
    const int padn = int(pad4(written) - written);
    if (g.rank() < padn && written + g.rank() < out_cap) out[written + g.rank()] = INT_MAX;
    g.sync();
    return written;
}

template <class G>
struct PathK;
template <>
struct PathK<WarpG> {
    static constexpr int K = 4;
};
template <int T>
struct PathK<BlockG<T>> {
    static constexpr int K = 8;
};

// Rank form while both lists fit in two rounds of the group (one binary
// search per element, all independent); merge-path beyond that, where the
// per-element searches would take many rounds.
template <class G, bool GA, bool GB>
__device__ __forceinline__ int merge_t(const G& g, const int32_t* a, int na, const int32_t* b, int nb, int32_t* out,
                                       int out_cap, int* err) {
    if ((na > nb ? na : nb) <= 2 * G::kSize) return xor_merge<G, GA, GB>(g, a, na, b, nb, out, out_cap, err);
    return xor_merge_path<G, PathK<G>::K, GA, GB>(g, a, na, b, nb, out, out_cap, err);
}

template <class G>
__device__ int merge(const G& g, const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb, int32_t* out,
                     int out_cap, int* err) {
#define SSPP_MG(A_, B_) merge_t<G, A_, B_>(g, a, na, b, nb, out, out_cap, err)
    return SSPP_DISPATCH2(ga, gb, SSPP_MG);
#undef SSPP_MG
}

// largest index of a xor b below their common top a[na-1] == b[nb-1]; -1 if none
__device__ __forceinline__ int next_low(const int32_t* a, int na, bool ga, const int32_t* b, int nb, bool gb) {
    int i = na - 2, j = nb - 2;
    while (i >= 0 && j >= 0) {
        int x = ldv(a + i, ga), y = ldv(b + j, gb);
        if (x != y) return x > y ? x : y;
        i--;
        j--;
    }
    if (i >= 0) return ldv(a + i, ga);
    if (j >= 0) return ldv(b + j, gb);
    return -1;
}

// global -> shared copy of int4 units [k0, k1) of a slot
template <class G>
__device__ __forceinline__ void copy4(const G& g, int32_t* dst, const int32_t* src, int k0, int k1) {
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = k0 + g.rank(); k < k1; k += G::kSize) d4[k] = __ldcg(s4 + k);
}

template <class G>
__device__ __forceinline__ void store4(const G& g, int32_t* dst, const int32_t* src, int n4) {
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
    int32_t* buf;      // current entries (shared memory, or the data part of an arena slot)
    int len;
    bool global;       // buf lives in the arena
    bool gpriv;        // buf is a private arena buffer (never published, reusable)
    int64_t gslot;     // arena slot of buf when global
    int64_t gcap;      // ints of that slot
    int64_t slot;      // arena slot of the published version
    bool dirty;        // differs from the published version
};

// Makes the working column the published version of `col`; false when the
// arena is exhausted.
template <class G>
__device__ bool publish(const G& g, const ReduceArgs& A, int col, Work& w) {
    int64_t so;
    if (w.global) {
        so = w.gslot;
        w.gpriv = false;  // published versions are immutable
    } else {
        so = alloc(g, A, slot_ints(w.len));
        if (so < 0) return false;
        store4(g, A.arena + so + kHdr, w.buf, int(pad4(w.len)) >> 2);
        if (g.leader()) cnt_add(&A.counters[CNT_PUBLISHED], (long long)slot_ints(w.len));
    }
    if (g.leader()) *reinterpret_cast<int4*>(A.arena + so) = make_int4(w.len, col, 0, 0);
    g.sync();
    if (g.leader()) {
        __threadfence();
        A.desc[col] = pack_desc(uint64_t(so), uint32_t(w.len));
    }
    w.slot = so;
    w.dirty = false;
    return true;
}

enum Outcome { OUT_OWNER, OUT_ZERO, OUT_PARKED, OUT_DEFERRED, OUT_FAIL };

// additions between two looks at a column's cleared flag
constexpr int kClearCheck = 64;

// Short addends in the CTA tier.  Along the long chains the CTA tier runs, the
// working column holds hundreds to thousands of entries while the addends
// (owners' versions) hold a handful, so rewriting the column for each addend
// would cost O(column) per addition.  Warp 0 alone keeps the column as a
// sorted bulk in shared memory plus a delta: up to 32 pending entries (sorted,
// one per lane, in registers) whose xor with the bulk is the column.  The
// lowest row only moves down, so it is always the larger of the two tops (equal
// tops cancel); an addition removes that top and toggles the addend's other
// entries in the delta (a ballot and a shuffle each).  The delta is folded
// into the bulk when it fills and when the warp stops, by rewriting the bulk
// from the lowest position a delta entry lands, one constant-shift segment per
// delta entry, through the spare buffer.  The rest of the CTA waits at one
// barrier.  The warp stops, leaving the step to the general path, when the row
// must be claimed (no owner, or a larger one), the column is empty or below the
// band, or the addend is longer than kShortAddend entries or would not fit.
// Returns the additions done, or -1 after a failed self-check.
constexpr int kShortAddend = 28;  // header + entries in one 32-lane load

struct FastState {
    unsigned long long e;
    long long add_ints;
    int len, L, adds, bad;
};

// a[0..nb) xor {dv on lanes 0..d-1, ascending} back into a; returns the new
// length (the caller keeps it within the buffer) and pads with INT_MAX.  One
// warp; tmp is a spare buffer of the same capacity.
__device__ int fold_delta(int32_t* a, int nb, int dv, int d, int32_t* tmp, int* err) {
    const int lane = threadIdx.x & 31;
    int pos = nb;
    bool fnd = false;
    if (lane < d) {
        pos = lower_bound_t<false>(a, nb, dv);
        fnd = pos < nb && lds(a + pos) == dv;
    }
    const int pmin = warp_min(pos);
    const unsigned fmask = __ballot_sync(kFull, lane < d && fnd);
    const unsigned imask = __ballot_sync(kFull, lane < d && !fnd);
    // segment j (j = -1 .. d-1) of the bulk suffix: from delta entry j's position
    // (past the entry it cancels) to the next delta entry's; its entries move by
    // the insertions minus the cancellations at or before it
    for (int j = -1; j < d; j++) {
        const int pj = j < 0 ? pmin : __shfl_sync(kFull, pos, j);
        const bool fj = j >= 0 && ((fmask >> j) & 1);
        const int lo = pj + (fj ? 1 : 0);
        const int hi = j + 1 < d ? __shfl_sync(kFull, pos, j + 1) : nb;
        const unsigned upto = j < 0 ? 0u : (j == 31 ? kFull : ((2u << j) - 1));
        const int shift = __popc(imask & upto) - __popc(fmask & upto);
        for (int i = lo + lane; i < hi; i += 32) {
            const int t = i - pmin + shift;
            tmp[t] = lds(a + i);
        }
    }
    if (lane < d && !fnd) {  // inserted delta entries land before the bulk entry at their position
        const unsigned lt = lanemask_lt();
        const int t = pos - pmin + __popc(imask & lt) - __popc(fmask & lt);
        tmp[t] = dv;
    }
    __syncwarp();
    const int outl = nb - pmin + __popc(imask) - __popc(fmask);
    for (int i = lane; i < outl; i += 32) a[pmin + i] = tmp[i];
    const int nn = pmin + outl;
    if (lane < int(pad4(nn) - nn)) a[nn + lane] = INT_MAX;
    __syncwarp();
    (void)err;
    return nn;
}

// Runs of additions.  Lane j keeps the bulk entry a[cb-1-j] (cb: the bulk
// length when the cache was filled) and that row's inline apparent column, all
// loaded at once.  While the current low is the bulk top at cache lane h and
// its owner is an inline apparent column, the additions of the bulk rows at
// lanes h, h+1, ... follow one another without a look at the column: row
// r_{i+1} is the next low after the additions of r_h..r_i exactly when every
// entry those addends toggle, and the delta's top, lie below r_{i+1} (equal
// would cancel it).  Such a run removes its rows from the bulk top at once and
// toggles the addends' other entries into the delta; no dependent load waits
// between its additions.
constexpr int kCacheRefill = 16;  // cache lanes used before the cache is filled again
#ifndef SSPP_FAST_PREFETCH
#define SSPP_FAST_PREFETCH 1
#endif
#ifndef SSPP_FAST_TOGGLE3
#define SSPP_FAST_TOGGLE3 0
#endif
#ifndef SSPP_FAST_PVPF
#define SSPP_FAST_PVPF 0
#endif

// Inline apparent columns of the delta's entries (SSPP_FAST_DAP): when an
// entry enters the delta, its row's inline column is copied asynchronously
// (cp.async) into a ring of shared-memory slots, and the entry's lane keeps
// the insertion index with it as entries shift.  When the delta's top becomes
// the lowest row, often many additions after it was inserted, its column is
// already in shared memory: no dependent global load on the chain.  Copies are
// committed once per addition (or run); a read waits only for the group its
// entry was inserted in, and each commit first lets all but the last two
// groups finish, so a slot is never reused while a copy to it is in flight
// (two groups hold at most 2 x 96 insertions, the ring has 256 slots).
#ifndef SSPP_FAST_DAP
#define SSPP_FAST_DAP 1
#endif
#ifndef SSPP_FAST_TOGGLE_EAGER
#define SSPP_FAST_TOGGLE_EAGER 1
#endif
constexpr int kDapSlots = 256;
static_assert(!(SSPP_FAST_DAP && SSPP_FAST_TOGGLE3), "the three-entry toggle does not carry insertion indices");

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// largest entry of an inline apparent column below its top (-1 if none)
__device__ __forceinline__ int app_max_below(int4 q) {
    return q.x <= 0 ? -1 : (q.x == 1 ? q.y : (q.x == 2 ? q.z : q.w));
}

template <int T>
__device__ int fast_adds(const BlockG<T>& g, const ReduceArgs& A, int32_t minrow, int col, Work& w, int& L,
                         uint64_t& e, int32_t* tmp, int32_t* sb, long long& adds, long long& add_ints,
                         int iters_left) {
    __shared__ FastState fs;
#if SSPP_FAST_DAP
    __shared__ int4 s_dap[kDapSlots];
#endif
    (void)sb;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int32_t* a = w.buf;
        int nb = w.len;         // bulk a[0..nb), ascending; its top is a[nb-1]
        int d = 0;              // delta: dv on lanes 0..d-1, ascending, INT_MAX above
        int dv = INT_MAX;
        int Lc = L, done = 0, bad = 0;
        bool top_in_bulk = true;  // Lc is a[nb-1] (else the delta's top)
        uint64_t ec = e;
        long long ai = 0;
        int n_inline = 0;
        // bulk cache: lane j holds cr = a[cb - 1 - j] and its inline apparent column ca
        int cb = -1;
        int cr = -1;
        int4 ca = make_int4(-1, 0, 0, 0);
        // inline apparent columns of the last addend's largest entries,
        // loaded while that addition runs: one of them is usually the next low
        int pf_row = -1;
        int4 pf_ap = make_int4(-1, 0, 0, 0);
        uint64_t pf_pv = kNoOwner;  // ... and their pivot entries (relaxed), for owners that are not inline
        bool have_pf_pv = false;    // ec_pf below holds the current low's prefetched entry
        uint64_t ec_pf = kNoOwner;
        int next_clear = kClearCheck;  // additions before the next look at the cleared flag
        bool have_e = true;  // ec is the pivot entry of Lc
#if SSPP_FAST_DAP
        int dslot = 0;  // insertion index of dv (lanes < d); its inline column is s_dap[dslot % kDapSlots]
        int nslot = 0;  // insertions so far
        int g_open = 0, g_last = 0, g_prev = 0;  // first insertion of the open, last and previous groups
        auto dap_commit = [&]() {
            cp_async_commit();
            cp_async_wait<2>();  // every group before the last two has landed
            g_prev = g_last;
            g_last = g_open;
            g_open = nslot;
        };
#endif
        // toggles x in the delta (a fold into the bulk when the delta is full
        // invalidates the bulk cache)
        // (both outcomes' ballots and shuffles are issued together before the
        // branch: they depend only on the delta, so their latencies overlap;
        // SSPP_FAST_TOGGLE_EAGER 0 keeps them in dependent order.  Measured at
        // 64^3: one block per dimension 5.38 -> 5.29 ms, the reference's block
        // sizes 5.33 -> 5.30 ms.  The warp tier's register path keeps the
        // dependent order: there the eager form spilled and measured slower)
        auto toggle = [&](int x) {
#if SSPP_FAST_TOGGLE_EAGER
            const unsigned eq = __ballot_sync(kFull, lane < d && dv == x);
            unsigned lt = __ballot_sync(kFull, lane < d && dv < x);
            const int nx = __shfl_down_sync(kFull, dv, 1);
            const int pv = __shfl_up_sync(kFull, dv, 1);
#if SSPP_FAST_DAP
            const int ns = __shfl_down_sync(kFull, dslot, 1);
            const int ps = __shfl_up_sync(kFull, dslot, 1);
#endif
            if (eq) {
                const int q = __ffs(eq) - 1;
                if (lane >= q) {
                    dv = lane + 1 < d ? nx : INT_MAX;
#if SSPP_FAST_DAP
                    dslot = ns;
#endif
                }
                d--;
            } else {
                if (d == 32) {  // full: the bulk absorbs the delta, then x goes in first
                    nb = fold_delta(a, nb, dv, d, tmp, A.err);
                    d = 0;
                    dv = INT_MAX;
                    cb = -1;
                    lt = 0;
                }
                const int q = __popc(lt);
                if (lane > q && lane <= d) {  // never after a fold (d == 0): pv is not stale there
                    dv = pv;
#if SSPP_FAST_DAP
                    dslot = ps;
#endif
                }
                if (lane == q) {
                    dv = x;
#if SSPP_FAST_DAP
                    dslot = nslot;
                    int4* dst = s_dap + (nslot & (kDapSlots - 1));
                    if (x >= 0 && x < A.ncols) cp_async16(dst, A.app + x);
                    else *dst = make_int4(-1, 0, 0, 0);
#endif
                }
#if SSPP_FAST_DAP
                nslot++;
#endif
                d++;
            }
#else
            const unsigned eq = __ballot_sync(kFull, lane < d && dv == x);
            if (eq) {
                const int q = __ffs(eq) - 1;
                const int nx = __shfl_down_sync(kFull, dv, 1);
#if SSPP_FAST_DAP
                const int ns = __shfl_down_sync(kFull, dslot, 1);
                if (lane >= q) {
                    dv = lane + 1 < d ? nx : INT_MAX;
                    dslot = ns;
                }
#else
                if (lane >= q) dv = lane + 1 < d ? nx : INT_MAX;
#endif
                d--;
            } else {
                if (d == 32) {  // full: the bulk absorbs the delta
                    nb = fold_delta(a, nb, dv, d, tmp, A.err);
                    d = 0;
                    dv = INT_MAX;
                    cb = -1;
                }
                const int q = __popc(__ballot_sync(kFull, lane < d && dv < x));
                const int pv = __shfl_up_sync(kFull, dv, 1);
#if SSPP_FAST_DAP
                const int ps = __shfl_up_sync(kFull, dslot, 1);
                if (lane > q && lane <= d) {
                    dv = pv;
                    dslot = ps;
                }
                if (lane == q) {
                    dv = x;
                    dslot = nslot;
                    int4* dst = s_dap + (nslot & (kDapSlots - 1));
                    if (x >= 0 && x < A.ncols) cp_async16(dst, A.app + x);
                    else *dst = make_int4(-1, 0, 0, 0);
                }
                nslot++;
#else
                if (lane > q && lane <= d) dv = pv;
                if (lane == q) dv = x;
#endif
                d++;
            }
#endif
        };
        // toggles up to three ascending entries x0 < x1 < x2 at once: entries
        // found in the delta are removed, the others inserted; every output
        // lane finds its source with bit counts and one shuffle gathers it
        auto toggle3 = [&](int q, int x0, int x1, int x2) {
            if (d + q > 32) {  // the bulk absorbs the delta first
                nb = fold_delta(a, nb, dv, d, tmp, A.err);
                d = 0;
                dv = INT_MAX;
                cb = -1;
            }
            const unsigned below_d = d >= 32 ? kFull : ((1u << d) - 1);
            unsigned del = 0;
            int e0 = 64, e1 = 64, e2 = 64;  // output slots of the inserted entries (64: not inserted)
            int ninsb = 0;                  // entries inserted so far (all smaller than the next one)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                if (j >= q) break;
                const int x = j == 0 ? x0 : (j == 1 ? x1 : x2);
                const unsigned eq = __ballot_sync(kFull, dv == x) & below_d;
                if (eq) {
                    del |= eq;
                } else {
                    const unsigned lt = __ballot_sync(kFull, dv < x) & below_d;
                    const int e = __popc(lt) - __popc(del & lt) + ninsb;
                    if (j == 0) e0 = e;
                    else if (j == 1) e1 = e;
                    else e2 = e;
                    ninsb++;
                }
            }
            // output lane t: an inserted entry, or the (t - inserted before t)-th kept entry
            const int kt = (e0 < lane) + (e1 < lane) + (e2 < lane);
            int src = lane - kt;
            unsigned dm = del;
            while (dm) {
                const int pdel = __ffs(dm) - 1;
                if (pdel > src) break;
                src++;
                dm &= dm - 1;
            }
            const int g = __shfl_sync(kFull, dv, src & 31);
            const int nd = d - __popc(del) + ninsb;
            int v = src < d ? g : INT_MAX;
            if (lane == e0) v = x0;
            else if (lane == e1) v = x1;
            else if (lane == e2) v = x2;
            dv = lane < nd ? v : INT_MAX;
            d = nd;
        };
        while (done < iters_left && nb + d > 0 && Lc >= minrow) {
            if (done >= next_clear) {  // cleared meanwhile: the general path stops the column
                next_clear = done + kClearCheck;
                unsigned c = 0;
                if (lane == 0) c = ld_acquire_u8(A.cleared + col);
                if (__shfl_sync(kFull, c, 0)) break;
            }
            // the inline apparent column of the current low: from the bulk
            // cache when the low is the bulk top, else one load
            have_pf_pv = false;  // set below only when the prefetch holds this low's entry
            int4 ap;
            int h = -1;
            if (top_in_bulk) {
                if (cb < 0 || cb - nb >= kCacheRefill) {
                    cb = nb;
                    const int idx = nb - 1 - lane;
                    cr = idx >= 0 ? lds(a + idx) : -1;
                    ca = (cr >= 0 && cr < A.ncols) ? __ldg(A.app + cr) : make_int4(-1, 0, 0, 0);
                }
                h = cb - nb;
                ap.x = __shfl_sync(kFull, ca.x, h);
                ap.y = __shfl_sync(kFull, ca.y, h);
                ap.z = __shfl_sync(kFull, ca.z, h);
                ap.w = __shfl_sync(kFull, ca.w, h);
                if (__shfl_sync(kFull, cr, h) != Lc) {  // self-check: the cache lane holds the bulk top
                    bad = 1;
                    break;
                }
            } else {
#if SSPP_FAST_DAP
                // the low is the delta's top (lane d - 1): its column is in the ring
                const int idx = __shfl_sync(kFull, dslot, d - 1);
                if (idx >= g_last) cp_async_wait<0>();
                else if (idx >= g_prev) cp_async_wait<1>();
                __syncwarp();
                ap = s_dap[idx & (kDapSlots - 1)];
#else
                const unsigned pm = __ballot_sync(kFull, pf_row == Lc);
                const int src = pm ? __ffs(pm) - 1 : 31;
                ap = pf_ap;
                if (!pm) {
                    ap = make_int4(-1, 0, 0, 0);
                    if (lane == 31 && Lc >= 0 && Lc < A.ncols) ap = __ldg(A.app + Lc);
                }
                ap.x = __shfl_sync(kFull, ap.x, src);
                ap.y = __shfl_sync(kFull, ap.y, src);
                ap.z = __shfl_sync(kFull, ap.z, src);
                ap.w = __shfl_sync(kFull, ap.w, src);
                have_pf_pv = pm != 0 && ap.x < 0 && SSPP_FAST_PREFETCH && SSPP_FAST_PVPF;
                if (have_pf_pv) ec_pf = __shfl_sync(kFull, (unsigned long long)pf_pv, src);
#endif
            }
            if (top_in_bulk && ap.x >= 0) {
                // a run from cache lane h: lane l (> h) joins while lanes h..l-1
                // all joined, its row has an inline apparent column, and the
                // delta top and every entry the run toggled so far lie below it
                const int td = d > 0 ? __shfl_sync(kFull, dv, d - 1) : -1;
                const bool mine = lane >= h && cr >= 0 && ca.x >= 0;
                int mx = mine ? app_max_below(ca) : -1;
                mx = mx > td ? mx : td;
                int M = mx;  // inclusive prefix max over lanes h..lane
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(kFull, M, o);
                    if (lane >= o && lane - o >= h) M = t > M ? t : M;
                }
                const int mprev = __shfl_up_sync(kFull, M, 1);   // prefix max up to lane - 1
                const int mcnt = mine ? ca.x : 0;
                // entries toggled by lanes h..lane (inclusive), for the capacity bound
                int csum = mcnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(kFull, csum, o);
                    if (lane >= o && lane - o >= h) csum += t;
                }
                const bool join = lane == h || (lane > h && mine && mprev < cr);
                const bool fits = nb + d + csum <= A.cap && lane - h < iters_left - done;
                const unsigned stop = __ballot_sync(kFull, lane >= h && !(join && fits));
                // lanes h .. first stopping lane - 1 form the run; lane h always
                // joins, so the run is empty only when lane h does not fit
                const unsigned above = stop & (kFull << h);
                const int end = above ? __ffs(above) - 1 : 32;
                const int P = end - h;
                if (P > 0) {
                    const int rlast = __shfl_sync(kFull, cr, end - 1);
                    nb -= P;
                    for (int i = h; i < end; i++) {
                        const int qx = __shfl_sync(kFull, ca.x, i);
                        const int qy = __shfl_sync(kFull, ca.y, i);
                        const int qz = __shfl_sync(kFull, ca.z, i);
                        const int qw = __shfl_sync(kFull, ca.w, i);
                        if (SSPP_FAST_TOGGLE3) {
                            if (qx > 0) toggle3(qx, qy, qz, qw);
                        } else {
                            if (qx > 0) toggle(qy);
                            if (qx > 1) toggle(qz);
                            if (qx > 2) toggle(qw);
                        }
                        ai += 2 * (nb + d) + qx + 2;
                    }
                    done += P;
                    n_inline += P;
                    pf_row = -1;
#if SSPP_FAST_DAP
                    dap_commit();
#endif
                    // the next lowest row: the larger top; equal tops cancel
                    int nl = -1;
                    while (true) {
                        const int tb = nb > 0 ? lds(a + nb - 1) : -1;
                        const int tdd = d > 0 ? __shfl_sync(kFull, dv, d - 1) : -1;
                        if (tb >= 0 && tb == tdd) {
                            nb--;
                            d--;
                            if (lane == d) dv = INT_MAX;
                            continue;
                        }
                        top_in_bulk = tb > tdd;
                        nl = top_in_bulk ? tb : tdd;
                        break;
                    }
                    if (nl >= rlast || nl >= A.ncols) {  // self-check: the lowest row only moves down
                        bad = 1;
                        break;
                    }
                    Lc = nl;
                    have_e = false;
                    ec = kNoOwner;  // unknown; the general path's claim retries with the real entry
                    continue;
                }
            }
            int plen, bj;
            if (ap.x >= 0) {  // apparent owner: permanent, its entries are at hand
                plen = ap.x + 1;
                bj = lane == 0 ? ap.y : (lane == 1 ? ap.z : ap.w);
            } else {
                if (!have_e) {
                    if (have_pf_pv) {
                        // read early (relaxed): an older entry still names an earlier
                        // column with this low, whose published versions never change;
                        // the fence orders the slot reads after it
                        ec = ec_pf;
                        __threadfence();
                    } else {
                        uint64_t t = 0;
                        if (lane == 0) t = ld_acquire_u64(A.pivot + Lc);
                        ec = __shfl_sync(kFull, (unsigned long long)t, 0);
                    }
                    have_e = true;
                }
                if (pv_col(ec) >= col) break;                         // claim: the general path
                if (pv_slot(ec) + kHdr > uint64_t(A.arena_cap)) break;  // the general path reports it
                const int v = __ldcg(A.arena + pv_slot(ec) + lane);      // header and the first 28 entries
                plen = __shfl_sync(kFull, v, 0);
                const int hcol = __shfl_sync(kFull, v, 1);
                if (plen < 1 || plen > kShortAddend || hcol != pv_col(ec)) break;
                if (__shfl_sync(kFull, v, (kHdr + plen - 1) & 31) != Lc) break;  // the general path reports it
                bj = __shfl_sync(kFull, v, (lane + kHdr) & 31);
            }
            const int m = plen - 1;  // addend entries below the common top
            if (nb + d + m > A.cap) break;  // the folded column might not fit
            // the addend's three largest other entries: their inline apparent
            // columns load while this addition runs
            pf_row = -1;
            if (SSPP_FAST_PREFETCH && !SSPP_FAST_DAP && lane < m && lane >= m - 3 && bj >= 0 && bj < A.ncols) {
                pf_row = bj;
                pf_ap = __ldg(A.app + bj);
                if (SSPP_FAST_PVPF) pf_pv = ld_relaxed_u64(A.pivot + bj);
            }
            if (top_in_bulk) {  // the tops cancel
                nb--;
            } else {
                d--;
                if (lane == d) dv = INT_MAX;
            }
            // toggle the addend's other entries in the delta
            if (SSPP_FAST_TOGGLE3 && ap.x >= 0) {
                if (m > 0) toggle3(m, ap.y, ap.z, ap.w);
            } else {
                for (int j = 0; j < m; j++) toggle(__shfl_sync(kFull, bj, j));
            }
#if SSPP_FAST_DAP
            dap_commit();
#endif
            // the next lowest row: the larger top; equal tops cancel
            int nl = -1;
            while (true) {
                const int tb = nb > 0 ? lds(a + nb - 1) : -1;
                const int td = d > 0 ? __shfl_sync(kFull, dv, d - 1) : -1;
                if (tb >= 0 && tb == td) {
                    nb--;
                    d--;
                    if (lane == d) dv = INT_MAX;
                    continue;
                }
                top_in_bulk = tb > td;
                nl = top_in_bulk ? tb : td;
                break;
            }
            ai += 2 * (nb + d) + plen + 1;
            done++;
            if (ap.x >= 0) n_inline++;
            if (nl >= Lc || nl >= A.ncols) {  // self-check: the lowest row only moves down
                bad = 1;
                break;
            }
            Lc = nl;
            have_e = false;
            ec = kNoOwner;  // unknown; the general path's claim retries with the real entry
        }
        if (d > 0) nb = fold_delta(a, nb, dv, d, tmp, A.err);
#if SSPP_FAST_DAP
        cp_async_wait<0>();  // no copy may land in the ring after this call
#endif
        if (lane == 0) {
            fs.len = nb;
            fs.L = nb > 0 ? lds(a + nb - 1) : -1;
            fs.e = ec;
            fs.adds = done;
            fs.add_ints = ai;
            fs.bad = bad || (fs.L != (nb > 0 ? Lc : -1) && done > 0);
            if (fs.bad) atomicOr(A.err, ERRB_CHECK);
            if (done) {
                cnt_add(&A.counters[CNT_FAST_INLINE], n_inline);
                cnt_add(&A.counters[CNT_FAST_SLOT], done - n_inline);
            }
        }
    }
    __syncthreads();
    const int done = fs.adds;
    if (fs.bad) return -1;
    if (done > 0) {
        w.len = fs.len;
        w.dirty = true;
        L = fs.L;
        e = fs.e;
        adds += done;
        add_ints += fs.add_ints;
    }
    __syncthreads();  // fs is rewritten by the next call
    return done;
}

// Warp tier, inline apparent addends.  A working column of at most 32 entries
// is held in registers, one entry per lane, ascending; while the owner of its
// lowest row is an inline apparent column (Device::app), an addition removes
// the top and toggles the addend's other entries in place (a ballot and a
// shuffle each), with no staging and no shared-memory merge, and the inline
// columns of the addend's entries load during the addition (one of them is
// usually the next low).  Stops at a row without such an owner, below the
// band, or when the column would outgrow 32 entries or the buffer; the column
// goes back to w.buf.  Returns the additions done, or -1 after a failed
// self-check.
#ifndef SSPP_WARP_REG
#define SSPP_WARP_REG 1
#endif
__device__ int warp_adds(const ReduceArgs& A, int32_t minrow, Work& w, int& L, uint64_t& e, int4 ap, long long& adds,
                         long long& add_ints, int iters_left) {
    const int lane = threadIdx.x & 31;
    int len = w.len;
    int ev = lane < len ? lds(w.buf + lane) : INT_MAX;
    int Lc = L, done = 0;
    bool bad = false;
    long long ai = 0;
    int pf_row = -1;
    int4 pf_ap = make_int4(-1, 0, 0, 0);
    while (done < iters_left && ap.x >= 0) {
        const int m = ap.x;
        if (len - 1 + m > 32 || len - 1 + m > A.cap) break;
        const int bj = lane == 0 ? ap.y : (lane == 1 ? ap.z : ap.w);
        pf_row = -1;
        if (lane < m && bj >= 0 && bj < A.ncols) {
            pf_row = bj;
            pf_ap = __ldg(A.app + bj);
        }
        len--;  // the tops cancel
        if (lane == len) ev = INT_MAX;
        for (int j = 0; j < m; j++) {
            const int x = j == 0 ? ap.y : (j == 1 ? ap.z : ap.w);
            const unsigned eq = __ballot_sync(kFull, lane < len && ev == x);
            if (eq) {
                const int q = __ffs(eq) - 1;
                const int nx = __shfl_down_sync(kFull, ev, 1);
                if (lane >= q) ev = lane + 1 < len ? nx : INT_MAX;
                len--;
            } else {
                const int q = __popc(__ballot_sync(kFull, lane < len && ev < x));
                const int pv = __shfl_up_sync(kFull, ev, 1);
                if (lane > q && lane <= len) ev = pv;
                if (lane == q) ev = x;
                len++;
            }
        }
        ai += 2 * len + m + 2;
        done++;
        const int nl = len > 0 ? __shfl_sync(kFull, ev, (len - 1) & 31) : -1;
        if (nl >= Lc) {  // self-check: the lowest row only moves down
            bad = true;
            break;
        }
        Lc = nl;
        if (Lc < 0 || Lc < minrow) break;
        const unsigned pm = __ballot_sync(kFull, pf_row == Lc);
        const int src = pm ? __ffs(pm) - 1 : 31;
        int4 q4 = pf_ap;
        if (!pm) {
            q4 = make_int4(-1, 0, 0, 0);
            if (lane == 31 && Lc < A.ncols) q4 = __ldg(A.app + Lc);
        }
        ap.x = __shfl_sync(kFull, q4.x, src);
        ap.y = __shfl_sync(kFull, q4.y, src);
        ap.z = __shfl_sync(kFull, q4.z, src);
        ap.w = __shfl_sync(kFull, q4.w, src);
    }
    if (bad) {
        if (lane == 0) atomicOr(A.err, ERRB_CHECK);
        return -1;
    }
    if (done > 0) {
        if (lane < pad4(len)) w.buf[lane] = lane < len ? ev : INT_MAX;
        __syncwarp();
        w.len = len;
        w.dirty = true;
        L = Lc;
        uint64_t t = kNoOwner;
        if (lane == 0 && Lc >= 0 && Lc >= minrow) t = ld_acquire_u64(A.pivot + Lc);
        e = __shfl_sync(kFull, (unsigned long long)t, 0);
        adds += done;
        add_ints += ai;
    }
    return done;
}

// Reduces column `col` until it owns its lowest row, becomes zero, or its
// lowest row drops below the band.  With `defer`, a column whose entries (or
// whose next addend or sum) exceed the shared capacity is published and
// returned as OUT_DEFERRED for the heavy tier; without it such columns continue
// in arena buffers.  *displaced receives the owner this column displaced (-1
// if none).  sp holds kHdr + cap ints (staged addend with its header).
template <class G>
__device__ Outcome reduce_column(const G& g, const ReduceArgs& A, const Band& band, int col, int32_t* sw0,
                                 int32_t* sw1, int32_t* sp, bool defer, int* displaced) {
    const int32_t minrow = band.minrow;
    *displaced = -1;
    uint64_t d = 0;
    if (g.leader()) d = ld_cg_u64(A.desc + col);
    d = g.bcast64(d);
    Work w;
    w.len = int(desc_len(d));
    w.slot = int64_t(desc_off(d));
    w.dirty = false;
    if (w.slot + slot_ints(w.len) > A.arena_cap) {  // self-check: descriptor inside the arena
        if (g.leader()) atomicOr(A.err, ERRB_CHECK);
        return OUT_FAIL;
    }
    if (w.len <= A.cap) {
        copy4(g, sw0, A.arena + w.slot + kHdr, 0, int(pad4(w.len)) >> 2);
        g.sync();
        w.buf = sw0;
        w.global = false;
        w.gslot = 0;
    } else if (defer) {
        return OUT_DEFERRED;
    } else {
        w.buf = A.arena + w.slot + kHdr;
        w.global = true;
        w.gslot = w.slot;
    }
    w.gpriv = false;
    w.gcap = 0;
    // a private arena buffer freed by the last merge, reused by the next one
    // that does not fit in shared memory (chains of long sums then need two
    // buffers, not one per addition)
    int64_t spare = -1, spare_cap = 0;
    long long adds = 0, add_ints = 0;
    Outcome res = OUT_FAIL;
    int L = w.len ? ldv(w.buf + w.len - 1, w.global) : -1;
    uint64_t e = kNoOwner;
    if (L >= A.ncols) {  // self-check: row index in range
        if (g.leader()) atomicOr(A.err, ERRB_CHECK);
        return OUT_FAIL;
    }
    // inline apparent column of row r (every thread loads it: one transaction per warp)
    auto app_of = [&](int r) { return (r >= 0 && r >= minrow) ? __ldg(A.app + r) : make_int4(-1, 0, 0, 0); };
    int4 apc = app_of(L);
    if (L >= minrow) {
        if (g.leader()) e = ld_acquire_u64(A.pivot + L);
        e = g.bcast64(e);
    }
    // speculative first staging round: header + as many entries as one pass of the group reads
    const int first4 = min(G::kSize, (kHdr + A.cap) >> 2);
    int next_check = 0;
    for (int iter = 0;; iter++) {
        if (iter >= next_check) {
            // Cleared meanwhile: a column of the next higher dimension claimed this
            // column's row, so the column is positive and zero once reduced (and a row
            // never loses its owner, so it stays cleared).  It owns no row now (a claim
            // ends the reduction), so it stops here as zero.
            next_check = iter + kClearCheck;
            int c = 0;
            if (g.leader()) c = int(ld_acquire_u8(A.cleared + col));
            if (g.bcast(c)) {
                if (g.leader()) {
                    A.desc[col] = pack_desc(0, 0);
                    A.low[col] = -1;
                }
                res = OUT_ZERO;
                break;
            }
        }
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
        if (L < minrow) {
            if (w.dirty && !publish(g, A, col, w)) break;
            if (g.leader()) A.low[col] = L;
            res = OUT_PARKED;
            break;
        }
        const int p = pv_col(e);
        if (p > col) {  // no owner, or a larger one: claim the row
            if (w.dirty && !publish(g, A, col, w)) break;
            uint64_t old = 0;
            if (g.leader()) {
                // the column's final state goes out before the claim: a group
                // that later displaces it writes its own state after this one
                const uint8_t was = A.state[col];
                A.low[col] = L;
                A.state[col] = ST_OWNER;
                __threadfence();
                old = atomicCAS(reinterpret_cast<unsigned long long*>(A.pivot + L), (unsigned long long)e,
                                (unsigned long long)pv_pack(col, uint64_t(w.slot)));
                if (old != e) A.state[col] = was;  // not claimed: still in progress here
            }
            old = g.bcast64(old);
            if (old == e) {
                if (g.leader()) {
                    if (e == kNoOwner) A.cleared[L] = 1;  // twist clearing of the positive row column
                    else cnt_add(&A.counters[CNT_DISPLACED], 1ll);
                }
                *displaced = (e == kNoOwner) ? -1 : p;
                res = OUT_OWNER;
                break;
            }
            e = old;  // someone else changed the owner; look again
            continue;
        }
        // looked at on every pass once the chain is long enough: the register
        // path adds many additions to iter at once, so iter seldom lands on a
        // multiple of the limit (a test on multiples misses most long chains;
        // measured at 64^3: 5.90 -> 5.38 ms per reduction with every pass)
        if (defer && band.drain_ctr && A.light_chain > 0 && iter >= A.light_chain) {
            // once the step's window is handed out, a long chain in the warp tier
            // only holds up the step's tail: the CTA tier continues it on a side
            // stream while the next step runs
            int drained = 0;
            if (g.leader()) drained = __ldcg(band.drain_ctr) >= band.drain_total;
            if (g.bcast(drained)) {
                if (w.dirty && !publish(g, A, col, w)) break;
                res = OUT_DEFERRED;
                break;
            }
        }
        if constexpr (G::kSize > 32) {  // CTA tier: short addends by one warp
            if (!w.global) {
                const int done = fast_adds(g, A, minrow, col, w, L, e, w.buf == sw0 ? sw1 : sw0, sp, adds, add_ints,
                                           kMaxMergesPerColumn - iter);
                if (done < 0) break;
                if (done > 0) {
                    iter += done;
                    apc = app_of(L);
                    continue;
                }
            }
        } else if (SSPP_WARP_REG) {  // warp tier: the column in registers
            if (!w.global && apc.x >= 0 && w.len <= 32) {
#ifndef SSPP_WARP_RUN_CAP
#define SSPP_WARP_RUN_CAP kClearCheck
#endif
                const int done = warp_adds(A, minrow, w, L, e, apc, adds, add_ints,
                                           min(SSPP_WARP_RUN_CAP, kMaxMergesPerColumn - iter));
                if (done < 0) break;
                if (done > 0) {
                    iter += done;
                    apc = app_of(L);
                    continue;
                }
            }
        }
        // add the owner's version (p < col, same lowest row): stage header + entries
        if (pv_slot(e) + kHdr > uint64_t(A.arena_cap)) {  // self-check: entry inside the arena
            if (g.leader()) atomicOr(A.err, ERRB_CHECK);
            break;
        }
        const int32_t* src = A.arena + pv_slot(e);
        int plen;
        if (apc.x >= 0) {  // apparent owner: its entries are inline, no arena read
            plen = apc.x + 1;
            if (g.leader()) {
                sp[kHdr] = apc.y;
                sp[kHdr + 1] = apc.z;
                sp[kHdr + 2] = apc.w;
                sp[kHdr + 3] = INT_MAX;
                sp[kHdr + apc.x] = L;
            }
            g.sync();
        } else {
            copy4(g, sp, src, 0, first4);
            g.sync();
            plen = sp[0];
            if (plen < 1 || plen > int(kMaxColLen) || sp[1] != p ||
                int64_t(pv_slot(e)) + slot_ints(plen) > A.arena_cap) {  // self-check: header of the owner's version
                if (g.leader()) atomicOr(A.err, ERRB_CHECK);
                break;
            }
        }
        const int32_t* pb;
        bool pg;
        if (apc.x >= 0) {
            pb = sp + kHdr;
            pg = false;
        } else if (plen <= A.cap) {
            const int n4 = (kHdr + int(pad4(plen))) >> 2;
            if (n4 > first4) {
                copy4(g, sp, src, first4, n4);
                g.sync();
            }
            pb = sp + kHdr;
            pg = false;
        } else if (defer) {
            if (w.dirty && !publish(g, A, col, w)) break;
            res = OUT_DEFERRED;
            break;
        } else {
            pb = src + kHdr;
            pg = true;
        }
        if (g.leader() && (plen == 0 || ldv(pb + plen - 1, pg) != L)) atomicOr(A.err, ERRB_BAD_INPUT);
        // the next lowest row is known before the merge: request its pivot entry now
        const int L2 = next_low(w.buf, w.len, w.global, pb, plen, pg);
        if (L2 >= A.ncols) {  // self-check: row index in range
            if (g.leader()) atomicOr(A.err, ERRB_CHECK);
            break;
        }
        // the group's last thread takes the entry: in short merges it holds no
        // element, so its acquire load completes while the others merge
        uint64_t pref = kNoOwner;
        if (g.rank() == G::kSize - 1 && L2 >= minrow && L2 >= 0) pref = ld_acquire_u64(A.pivot + L2);
        const int4 apn = app_of(L2);
        int out_len;
        const int bound = w.len + plen - 2;
        if (bound <= A.cap) {
            int32_t* dst = (w.global || w.buf == sw1) ? sw0 : sw1;
            out_len = merge(g, w.buf, w.len, w.global, pb, plen, pg, dst, A.cap, A.err);
            if (w.global && w.gpriv) {
                spare = w.gslot;
                spare_cap = w.gcap;
            }
            w.buf = dst;
            w.global = false;
        } else {
            const int common = count_common(g, w.buf, w.len, w.global, pb, plen, pg);
            out_len = w.len + plen - 2 * common;
            if (out_len > int(kMaxColLen)) {
                if (g.leader()) atomicOr(A.err, ERRB_LEN);
                break;
            }
            if (out_len <= A.cap) {
                int32_t* dst = (w.global || w.buf == sw1) ? sw0 : sw1;
                merge(g, w.buf, w.len, w.global, pb, plen, pg, dst, A.cap, A.err);
                if (w.global && w.gpriv) {
                    spare = w.gslot;
                    spare_cap = w.gcap;
                }
                w.buf = dst;
                w.global = false;
            } else if (defer) {
                if (w.dirty && !publish(g, A, col, w)) break;
                res = OUT_DEFERRED;
                break;
            } else {
                const int64_t need = slot_ints(out_len);
                int64_t so, cap_so;
                if (spare >= 0 && spare_cap >= need) {
                    so = spare;
                    cap_so = spare_cap;
                    spare = -1;
                } else {
                    cap_so = (need + (need >> 1) + 3) & ~int64_t(3);  // slack for a growing sum
                    so = alloc(g, A, cap_so);
                    if (so < 0) break;
                    if (g.leader()) cnt_add(&A.counters[CNT_PUBLISHED], (long long)cap_so);
                }
                merge(g, w.buf, w.len, w.global, pb, plen, pg, A.arena + so + kHdr, int(pad4(out_len)), A.err);
                if (w.global && w.gpriv) {
                    spare = w.gslot;
                    spare_cap = w.gcap;
                }
                w.buf = A.arena + so + kHdr;
                w.global = true;
                w.gpriv = true;
                w.gslot = so;
                w.gcap = cap_so;
            }
        }
        adds++;
        add_ints += w.len + plen + out_len;
        w.len = out_len;
        w.dirty = true;
        L = L2;
        e = g.bcast64_last(pref);
        apc = apn;
    }
    if (g.leader() && adds) {
        cnt_add(&A.counters[CNT_ADDITIONS], adds);
        cnt_add(&A.counters[CNT_ADD_INTS], add_ints);
        if (!defer) cnt_add(&A.counters[CNT_HEAVY_ADDS], adds);
    }
    return res;
}

// Final state of a column after reduce_column; returns false on failure.
template <class G>
__device__ __forceinline__ bool settle(const G& g, const ReduceArgs& A, int col, Outcome o) {
    if (g.leader()) {
        switch (o) {
            case OUT_OWNER: break;  // written before the claim
            case OUT_ZERO: A.state[col] = ST_ZERO; break;
            case OUT_DEFERRED: {
                A.state[col] = ST_HEAVY;
                int i = atomicAdd(A.pool_tail, 1);
                if (i < A.pool_cap) A.heavy[i] = col;
                else atomicOr(A.err, ERRB_CAPACITY);  // pool full: the run is repeated with a larger one
                break;
            }
            default: __threadfence(); st_release_u8(A.state + col, ST_ACTIVE); break;  // parked / failed
        }
    }
    g.sync();
    return o != OUT_FAIL;
}

// The runnable columns of a step: window entries that are active, not cleared
// and whose lowest row lies in the band (low >= minrow), listed in window
// order within each block (one atomic per block pass) and counted in ctr[5].
// One thread per entry reads the flags with independent loads, so the warp
// tier then takes runnable columns one at a time instead of walking the whole
// window with a shared counter.  A flag set concurrently (a cleared flag from
// the previous dimension's CTA tier) is read again by the warp tier.
constexpr int kFilterThreads = 256;

__global__ void __launch_bounds__(kFilterThreads) k_light_filter(const int32_t* active, int32_t beg, int32_t end,
                                                                 int32_t minrow, const uint8_t* state,
                                                                 const uint8_t* cleared, const int32_t* low,
                                                                 int32_t* out, int* ctr) {
    __shared__ int s_warp[kFilterThreads / 32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t b0 = beg + int64_t(blockIdx.x) * kFilterThreads; b0 < end; b0 += int64_t(gridDim.x) * kFilterThreads) {
        const int64_t i = b0 + threadIdx.x;
        int32_t c = -1;
        bool r = false;
        if (i < end) {
            c = __ldcs(active + i);
            r = __ldcg(state + c) == ST_ACTIVE && !__ldcg(cleared + c) && __ldcg(low + c) >= minrow;
        }
        const unsigned m = __ballot_sync(kFull, r);
        if (lane == 0) s_warp[wid] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < kFilterThreads / 32; w++) {
                const int x = s_warp[w];
                s_warp[w] = t;
                t += x;
            }
            s_base = t ? atomicAdd(ctr + 5, t) : 0;
        }
        __syncthreads();
        if (r) out[s_base + s_warp[wid] + __popc(m & ((1u << lane) - 1))] = c;
        __syncthreads();  // s_warp and s_base are rewritten by the next pass
    }
}

// The last warp-tier block of a step to finish marks the step's slice of the
// CTA-tier pool: it ends at the pool tail, where the next step's slice starts
// (every deferral of the step is appended before its block finishes).
__device__ void light_block_done(const ReduceArgs& A) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(A.ctr + 4, 1) == int(gridDim.x) - 1) {
            __threadfence();
            const int t = ld_acquire(A.pool_tail);
            A.ctr[2] = t;
            if (A.ctr_next) A.ctr_next[1] = t;
        }
    }
}

// Light tier: warps take `chunk` window entries at a time and reduce the
// runnable ones (active, not cleared, lowest row inside the band).
// At least 9 blocks per SM: the compiler then keeps the kernel at 56 registers
// with nothing spilled (left free, it spilled 16 bytes at the same count);
// measured 64^3 5.79 -> 5.60 ms per reduction.
#ifndef SSPP_LIGHT_MIN_BLOCKS
#define SSPP_LIGHT_MIN_BLOCKS 9
#endif
__global__ void __launch_bounds__(128, SSPP_LIGHT_MIN_BLOCKS) k_reduce_light(ReduceArgs A) {
    extern __shared__ __align__(16) int32_t smem[];
    WarpG g;
    const int lane = g.rank();
    int32_t* sw0 = smem + size_t(threadIdx.x >> 5) * (3 * A.cap + kHdr);
    int32_t* sw1 = sw0 + A.cap;
    int32_t* sp = sw1 + A.cap;
    const int count = A.count ? __ldcg(A.count) : A.end - A.beg;
    const int end = A.beg + count;
    const int chunk = A.chunk;
    const Band band{A.minrow, A.ctr, count};
    bool stop = false;  // warp-uniform: a failure ends this warp's work
    while (!stop) {
        int base = 0;
        if (lane == 0) base = atomicAdd(A.ctr, chunk);
        base = g.bcast(base);
        if (base >= count) break;
        const int idx = A.beg + base + lane;
        int c = -1;
        bool run = false;
        if (lane < chunk && idx < end) {
            c = A.active[idx];
            run = ld_acquire_u8(A.state + c) == ST_ACTIVE && !ld_acquire_u8(A.cleared + c) &&
                  __ldcg(A.low + c) >= A.minrow;
        }
        unsigned m = __ballot_sync(kFull, run);
        while (m && !stop) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            int col = __shfl_sync(kFull, c, src);
            while (col >= 0) {  // the column, then any owner it displaced
                int next = -1;
                Outcome o = reduce_column(g, A, band, col, sw0, sw1, sp, true, &next);
                if (!settle(g, A, col, o)) {
                    stop = true;
                    break;
                }
                col = next;
            }
        }
    }
    light_block_done(A);
}

// Heavy tier: one CTA per deferred column, buffers of the level-2 capacity.
// Like the reference's block phase (include/kernel.h:966-1060) it does not
// stop at the band: a column handed over is reduced until it owns its lowest
// row or becomes zero.
template <int T>
__global__ void __launch_bounds__(T, 1) k_reduce_heavy(ReduceArgs A) {
    extern __shared__ __align__(16) int32_t smem[];
    __shared__ int gsm[2 * (T / 32 + 2)];
    __shared__ unsigned long long gsb[2];
    BlockG<T> g;
    g.sm = gsm;
    g.sb = gsb;
    int32_t* sw0 = smem;
    int32_t* sw1 = sw0 + A.cap;
    int32_t* sp = sw1 + A.cap;
    const int hb = __ldcg(A.ctr + 1), he = __ldcg(A.ctr + 2);
    const Band band{INT32_MIN, nullptr, 0};
    while (true) {
        int k = 0;
        if (g.leader()) k = hb + atomicAdd(A.ctr + 3, 1);
        k = g.bcast(k);
        if (k >= he) break;
        int col = __ldcg(A.heavy + k);
        while (col >= 0) {
            int next = -1;
            Outcome o = reduce_column(g, A, band, col, sw0, sw1, sp, false, &next);
            if (!settle(g, A, col, o)) return;
            col = next;
        }
        if (g.leader() && A.heavy_done) {  // progress for the host's dimension gate
            const int v = atomicAdd(A.heavy_done, 1) + 1;
            if (A.gate_host) st_relaxed_sys(A.gate_host, v);
        }
    }
}

// ------------------------------------------------------------- work queue
// One persistent, cooperative launch drains the (complex, block) items of a
// whole schedule: every spectral-sequence block of every complex of a batch
// (one complex when not batched), in each complex's own block order, with
// each complex's own dimension gate.  The host loop it replaces issues, per
// block, a warp-tier launch and a CTA-tier launch and synchronises at every
// dimension (the reference: include/specseq.h:616-661, three launches and a
// host synchronisation per block).
//
// Blocks [0, heavy_ctas) reduce the columns the warp tier defers, taken from a
// pool in order; the other blocks run independent warps over the open items.
// An item opens when its predecessor of the same complex has finished; the
// first item of a complex's next dimension opens once at most gate_left of the
// complex's CTA-tier columns are left (none for its last item, after which the
// complex is finished).  An item's entries are the columns its predecessors
// parked (their lowest row below the band; kept with that row, so a later
// block looks at a parked column without loading it) followed by the columns
// its block adds to the window; a warp takes `chunk` of them at a time.
// Columns of different complexes never share rows, so the items of different
// complexes run concurrently.  All blocks are resident (cooperative launch),
// so a block may poll for work that another block produces; every poll is
// bounded by spin_limit, after which the launch sets ERRB_TIMEOUT and leaves.

__device__ __forceinline__ int ld_acq(const int* p) { return ld_acquire(p); }
__device__ __forceinline__ void st_rel(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void queue_fail(const ReduceArgs& A, const QueueArgs& Q, int bits) {
    atomicOr(A.err, bits);
    st_rel(Q.abort, 1);
}

// Opens complex c's next item once its CTA-tier columns allow (c waits at a
// gate, its current item ci finished); any lane may call it.
__device__ void queue_try_gate(const QueueArgs& Q, int c, int ci) {
    const bool last = ci + 1 >= Q.item_end[c];
    if (ld_acq(Q.hpend + c) > (last ? 0 : Q.gate_left)) return;
    if (atomicCAS(Q.gate + c, 1, 0) != 1) return;
    if (last) {
        st_rel(Q.cur + c, -1);
        __threadfence();
        atomicAdd(Q.finished, 1);
    } else {
        st_rel(Q.cur + c, ci + 1);
    }
}

// Item `it` of complex c has finished: the next item opens, or, after the
// last block of a dimension, the complex waits at its gate.
__device__ __forceinline__ void queue_finish_item(const QueueArgs& Q, int c, int it, int flags) {
    __threadfence();
    if (flags & QF_LAST_OF_DIM) st_rel(Q.gate + c, 1);
    else st_rel(Q.cur + c, it + 1);
}

// Final state of a warp-tier column taken from the queue (settle's rules;
// deferred columns go to the pool, parked ones to the next item's list).
__device__ bool settle_q(const ReduceArgs& A, const QueueArgs& Q, int cc, int col, Outcome o, int it, int2* lout,
                         int32_t lcap) {
    bool ok = true;
    if ((threadIdx.x & 31) == 0) {
        switch (o) {
            case OUT_OWNER: break;
            case OUT_ZERO: A.state[col] = ST_ZERO; break;
            case OUT_DEFERRED: {
                A.state[col] = ST_HEAVY;
                atomicAdd(Q.hpend + cc, 1);
                const int i = atomicAdd(Q.pool_tail, 1);
                if (i < Q.pool_cap) {
                    Q.pool_c[i] = cc;
                    __threadfence();
                    st_rel(Q.pool + i, col);
                } else {
                    queue_fail(A, Q, ERRB_CAPACITY);  // the run is repeated with a larger pool
                }
                break;
            }
            case OUT_PARKED: {
                const int low = A.low[col];
                __threadfence();
                st_release_u8(A.state + col, ST_ACTIVE);
                const int j = atomicAdd(Q.lin + it + 1, 1);
                if (j < lcap) lout[j] = make_int2(col, low);
                else queue_fail(A, Q, ERRB_CAPACITY);
                break;
            }
            default:
                __threadfence();
                st_release_u8(A.state + col, ST_ACTIVE);
                queue_fail(A, Q, ERRB_CHECK);
                ok = false;
                break;
        }
    }
    __syncwarp();
    return __shfl_sync(kFull, ok ? 1 : 0, 0) != 0;
}

__device__ void queue_light(const ReduceArgs& A, const QueueArgs& Q, int32_t* sw0, int32_t* sw1, int32_t* sp,
                            int warps_per_block) {
    WarpG g;
    const int lane = g.rank();
    const int wl = (blockIdx.x - Q.heavy_ctas) * warps_per_block + (threadIdx.x >> 5);
    int start = Q.ncplx > 0 ? wl % Q.ncplx : 0;
    long long idle = 0;
    while (true) {
        int stop = 0;
        if (lane == 0) stop = ld_acq(Q.abort) || ld_acq(Q.finished) >= Q.ncplx;
        if (__shfl_sync(kFull, stop, 0)) break;
        // an open item with entries left: the lanes look at 32 complexes at a time
        int it = -1, cc = -1;
        for (int base = 0; base < Q.ncplx && it < 0; base += 32) {
            int myit = -1, c = -1;
            if (base + lane < Q.ncplx) {
                c = (start + base + lane) % Q.ncplx;
                const int ci = ld_acq(Q.cur + c);
                if (ci >= 0) {
                    if (ld_acq(Q.gate + c)) {
                        queue_try_gate(Q, c, ci);
                    } else {
                        const QItem& I = Q.items[ci];
                        const int total = ld_acq(Q.lin + ci) + (I.nend - I.nbeg);
                        if (total == 0) {  // nothing to do: whoever sees it first finishes it
                            if (atomicCAS(Q.taken + ci, 0, 1) == 0) queue_finish_item(Q, c, ci, I.flags);
                        } else if (__ldcg(Q.taken + ci) < total) {
                            myit = ci;
                        }
                    }
                }
            }
            const unsigned m = __ballot_sync(kFull, myit >= 0);
            if (m) {
                const int src = __ffs(m) - 1;
                it = __shfl_sync(kFull, myit, src);
                cc = __shfl_sync(kFull, c, src);
            }
        }
        if (it < 0) {
            if (++idle > Q.spin_limit) {
                if (lane == 0) queue_fail(A, Q, ERRB_TIMEOUT);
                break;
            }
            __nanosleep(256);
            continue;
        }
        idle = 0;
        start = cc;
        const QItem I = Q.items[it];
        const int nl = ld_acq(Q.lin + it);
        const int total = nl + (I.nend - I.nbeg);
        int base = 0;
        if (lane == 0) base = atomicAdd(Q.taken + it, Q.chunk);
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) continue;
        const int cnt = min(Q.chunk, total - base);
        const int32_t lcap = Q.list_cap[cc];
        const int2* lin_list = Q.lists + Q.list_off[cc] + ((I.flags & QF_HALF) ? lcap : 0);
        int2* lout = Q.lists + Q.list_off[cc] + ((I.flags & QF_HALF) ? 0 : lcap);
        int col = -1, lowc = 0;
        bool run = false, park = false;
        if (lane < cnt) {
            const int e = base + lane;
            if (e < nl) {
                const int2 v = lin_list[e];
                col = v.x;
                lowc = v.y;
            } else {
                col = A.active[I.nbeg + (e - nl)];
                lowc = __ldcg(A.low + col);
            }
            if (col < 0 || col >= A.ncols) {  // self-check: a list or active entry in range
                queue_fail(A, Q, ERRB_CHECK);
                col = -1;
            } else {
                const bool act = ld_acquire_u8(A.state + col) == ST_ACTIVE && !ld_acquire_u8(A.cleared + col);
                run = act && lowc >= I.minrow;
                park = act && lowc < I.minrow;
            }
        }
        // still below the band: on to the next item's list as they are
        const unsigned pm = __ballot_sync(kFull, park);
        if (pm) {
            int pb = 0;
            if (lane == 0) pb = atomicAdd(Q.lin + it + 1, __popc(pm));
            pb = __shfl_sync(kFull, pb, 0);
            if (park) {
                const int j = pb + __popc(pm & lanemask_lt());
                if (j < lcap) lout[j] = make_int2(col, lowc);
                else queue_fail(A, Q, ERRB_CAPACITY);
            }
        }
        const Band band{I.minrow, Q.taken + it, total};
        unsigned m = __ballot_sync(kFull, run);
        bool failed = false;
        while (m && !failed) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            int c2 = __shfl_sync(kFull, col, src);
            while (c2 >= 0) {  // the column, then any owner it displaced
                int next = -1;
                const Outcome o = reduce_column(g, A, band, c2, sw0, sw1, sp, true, &next);
                if (!settle_q(A, Q, cc, c2, o, it, lout, lcap)) {
                    failed = true;
                    break;
                }
                c2 = next;
            }
        }
        if (failed) break;
        // the chunk is finished; the warp finishing the item opens the next one
        int fin = 0;
        if (lane == 0) {
            __threadfence();
            fin = atomicAdd(Q.done + it, cnt) + cnt == total;
            if (fin) queue_finish_item(Q, cc, it, I.flags);
        }
        __syncwarp();
    }
}

template <int T>
__device__ void queue_heavy(const ReduceArgs& A, const QueueArgs& Q, const BlockG<T>& g, int32_t* sw0, int32_t* sw1,
                            int32_t* sp) {
    const Band band{INT32_MIN, nullptr, 0};
    long long idle = 0;
    while (true) {
        unsigned long long pk = 0;  // bit 63: stop; else (complex << 32) | column, or all ones for none
        if (g.leader()) {
            if (ld_acq(Q.abort) || ld_acq(Q.finished) >= Q.ncplx) {
                pk = 1ull << 63;
            } else {
                pk = ~0ull >> 1;
                const int h = ld_acq(Q.pool_head);
                if (h < Q.pool_cap) {
                    const int v = ld_acq(Q.pool + h);
                    if (v >= 0 && atomicCAS(Q.pool_head, h, h + 1) == h)
                        pk = (uint64_t(uint32_t(Q.pool_c[h])) << 32) | uint32_t(v);
                }
            }
        }
        pk = g.bcast64(pk);
        if (pk >> 63) break;
        if (pk == (~0ull >> 1)) {
            if (++idle > Q.spin_limit) {
                if (g.leader()) queue_fail(A, Q, ERRB_TIMEOUT);
                break;
            }
            if (g.leader()) __nanosleep(512);
            continue;
        }
        idle = 0;
        const int cc = int(pk >> 32);
        int col = int(uint32_t(pk));
        while (col >= 0) {
            int next = -1;
            const Outcome o = reduce_column(g, A, band, col, sw0, sw1, sp, false, &next);
            if (!settle(g, A, col, o)) {
                if (g.leader()) queue_fail(A, Q, ERRB_CHECK);
                return;
            }
            col = next;
        }
        if (g.leader()) {
            __threadfence();
            atomicSub(Q.hpend + cc, 1);
        }
    }
}

// Al: warp-tier arguments (cap = level-1 capacity), Ah: CTA tier (level 2).
template <int T>
__global__ void __launch_bounds__(T, 1) k_reduce_queue(ReduceArgs Al, ReduceArgs Ah, QueueArgs Q) {
    extern __shared__ __align__(16) int32_t smem[];
    __shared__ int gsm[2 * (T / 32 + 2)];
    __shared__ unsigned long long gsb[2];
    if (int(blockIdx.x) < Q.heavy_ctas) {
        BlockG<T> g;
        g.sm = gsm;
        g.sb = gsb;
        queue_heavy<T>(Ah, Q, g, smem, smem + Ah.cap, smem + 2 * Ah.cap);
    } else {
        int32_t* sw0 = smem + size_t(threadIdx.x >> 5) * (3 * Al.cap + kHdr);
        queue_light(Al, Q, sw0, sw0 + Al.cap, sw0 + 2 * Al.cap, T / 32);
    }
}

// per complex and dimension: active columns, min first row over non-empty
// columns and max low + 1 over active columns (the quantities ColumnShrink
// computes for the whole matrix, include/specseq.h:374-398)
__global__ void k_queue_info(int64_t n, int32_t k, const int64_t* cstart, const int32_t* perm, const int32_t* rdim,
                             const int32_t* arena, const uint64_t* desc, const int32_t* low, const uint8_t* state,
                             int32_t* act_cnt, int32_t* min_row, int32_t* max_row) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t d = desc[i];
        const uint32_t len = desc_len(d);
        if (!len) continue;
        const int64_t x = perm[i];
        int32_t a = 0, b = k;  // largest a with cstart[a] <= x
        while (b - a > 1) {
            const int32_t mid = (a + b) >> 1;
            if (cstart[mid] <= x) a = mid;
            else b = mid;
        }
        const int dm = rdim[i];
        const int64_t slot = int64_t(a) * kNumDims + dm;
        atomicMin(min_row + slot, arena[desc_off(d) + kHdr]);
        if (state[i] == ST_ACTIVE) {
            atomicAdd(act_cnt + slot, 1);
            atomicMax(max_row + slot, low[i] + 1);
        }
    }
}

int queue_complex_info(const Device& D, int32_t k, const int64_t* d_cstart, int32_t* act_cnt, int32_t* min_row,
                       int32_t* max_row, cudaStream_t s) {
    const int64_t m = int64_t(k) * kNumDims;
    cudaMemsetAsync(act_cnt, 0, sizeof(int32_t) * m, s);
    fill_i32(min_row, INT32_MAX, m, s);
    fill_i32(max_row, -1, m, s);
    if (D.n == 0) return 0;
    int64_t g = (D.n + 255) / 256;
    if (g > 65536) g = 65536;
    k_queue_info<<<unsigned(g), 256, 0, s>>>(D.n, k, d_cstart, D.perm, D.dim, D.arena, D.desc, D.low, D.state, act_cnt,
                                             min_row, max_row);
    return 3;
}

int light_smem_bytes(int cap) { return 4 * (3 * cap + kHdr) * 4; }
int heavy_smem_bytes(int cap) { return (3 * cap + kHdr) * 4; }

// Warp-tier additions per column after which, once its step's window is
// fully handed out, the column moves to the CTA tier: a step's light launch
// lasts as long as its longest chain, while CTA-tier launches overlap later
// steps on side streams.  Handing chains over while the window still has work
// would only move parallel work onto the (fewer) CTAs.
#ifndef SSPP_LIGHT_CHAIN
#define SSPP_LIGHT_CHAIN 8
#endif
constexpr int32_t kLightChain = SSPP_LIGHT_CHAIN;

static ReduceArgs make_args(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                            int chunk, int* ctr) {
    ReduceArgs A;
    A.ncols = int32_t(D.n);
    A.active = active;
    A.beg = beg;
    A.end = end;
    A.minrow = minrow;
    A.cap = cap;
    A.chunk = chunk;
    A.arena = D.arena;
    A.arena_cap = D.arena_cap;
    A.arena_top = D.arena_top;
    A.desc = D.desc;
    A.low = D.low;
    A.pivot = D.pivot;
    A.state = D.state;
    A.cleared = D.cleared;
    A.ctr = ctr;
    A.ctr_next = nullptr;
    A.count = nullptr;
    A.heavy = D.heavy;
    A.pool_tail = D.pool_tail;
    A.heavy_done = D.heavy_done;
    A.gate_host = D.gate_host;
    A.pool_cap = D.pool_cap;
    A.err = D.err;
    A.counters = D.counters;
    A.light_chain = kLightChain;
    A.app = D.app;
    return A;
}

void reduce_light_launch(const Device& D, const int32_t* active, int32_t beg, int32_t end, int32_t minrow, int cap,
                         int chunk, int* ctr, int* ctr_next, int grid, cudaStream_t s) {
    ReduceArgs A = make_args(D, active, beg, end, minrow, cap, chunk, ctr);
    A.ctr_next = ctr_next;
    k_reduce_light<<<grid, 128, light_smem_bytes(cap), s>>>(A);
}

void reduce_light_filtered_launch(const Device& D, int32_t beg, int32_t end, int32_t minrow, int cap, int chunk,
                                  int* ctr, int* ctr_next, int filter_grid, int grid, cudaStream_t s) {
    k_light_filter<<<filter_grid, kFilterThreads, 0, s>>>(D.active, beg, end, minrow, D.state, D.cleared, D.low,
                                                          D.runlist, ctr);
    ReduceArgs A = make_args(D, D.runlist, 0, 0, minrow, cap, chunk, ctr);
    A.ctr_next = ctr_next;
    A.count = ctr + 5;
    k_reduce_light<<<grid, 128, light_smem_bytes(cap), s>>>(A);
}

void reduce_heavy_launch(const Device& D, int cap, int threads, int* ctr, int grid, cudaStream_t s) {
    ReduceArgs A = make_args(D, nullptr, 0, 0, INT32_MIN, cap, 1, ctr);
    if (threads == 256) k_reduce_heavy<256><<<grid, 256, heavy_smem_bytes(cap), s>>>(A);
    else k_reduce_heavy<128><<<grid, 128, heavy_smem_bytes(cap), s>>>(A);
}

// The dynamic shared-memory limit is a property of the kernel (per device),
// shared by every context of the process: contexts with different capacities
// (the server's workers, each autotuned) only ever raise it, under a lock, so
// that no launch finds it lowered below its own request.
static cudaError_t raise_smem_limit(const void* fn, int slot, int bytes) {
    static std::mutex mu;
    static int limit[64][5] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> l(mu);
    int& cur = limit[dev & 63][slot];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

static int queue_smem_bytes(int cap1, int cap2, int threads) {
    const int light = (threads / 32) * (3 * cap1 + kHdr) * 4;
    const int heavy = (3 * cap2 + kHdr) * 4;
    return light > heavy ? light : heavy;
}

cudaError_t queue_configure(int cap1, int cap2, int threads, int* blocks_per_sm) {
    const int smem = queue_smem_bytes(cap1, cap2, threads);
    *blocks_per_sm = 0;
    cudaError_t e;
    if (threads == 256) {
        e = raise_smem_limit(reinterpret_cast<const void*>(k_reduce_queue<256>), 3, smem);
        if (e != cudaSuccess) return e;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_reduce_queue<256>, 256, smem);
    }
    e = raise_smem_limit(reinterpret_cast<const void*>(k_reduce_queue<128>), 4, smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_reduce_queue<128>, 128, smem);
}

cudaError_t reduce_queue_launch(const Device& D, int cap1, int cap2, int threads, const QueueArgs& Q, int grid,
                                cudaStream_t s) {
    ReduceArgs Al = make_args(D, D.active, 0, 0, INT32_MIN, cap1, 1, nullptr);
    ReduceArgs Ah = make_args(D, nullptr, 0, 0, INT32_MIN, cap2, 1, nullptr);
    Al.gate_host = Ah.gate_host = nullptr;
    Al.heavy_done = Ah.heavy_done = nullptr;
    QueueArgs q = Q;
    void* args[] = {&Al, &Ah, &q};
    const int smem = queue_smem_bytes(cap1, cap2, threads);
    if (threads == 256)
        return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_reduce_queue<256>), grid, 256, args, smem, s);
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_reduce_queue<128>), grid, 128, args, smem, s);
}

cudaError_t reduce_configure(int cap1, int cap2, int heavy_threads, int* light_blocks_per_sm,
                             int* heavy_blocks_per_sm) {
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k_reduce_light), 0, light_smem_bytes(cap1));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(light_blocks_per_sm, k_reduce_light, 128, light_smem_bytes(cap1));
    if (e != cudaSuccess) return e;
    if (heavy_threads == 256) {
        e = raise_smem_limit(reinterpret_cast<const void*>(k_reduce_heavy<256>), 1, heavy_smem_bytes(cap2));
        if (e != cudaSuccess) return e;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(heavy_blocks_per_sm, k_reduce_heavy<256>, 256,
                                                             heavy_smem_bytes(cap2));
    }
    e = raise_smem_limit(reinterpret_cast<const void*>(k_reduce_heavy<128>), 2, heavy_smem_bytes(cap2));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(heavy_blocks_per_sm, k_reduce_heavy<128>, 128,
                                                         heavy_smem_bytes(cap2));
}

}  // namespace sspp
