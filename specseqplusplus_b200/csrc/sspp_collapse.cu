// Flag-complex edge collapse (model bit 2).
//
// Reference counterparts: the graph build with edge filtration = edge order
// (include/specseq.h:209-212), GUDHI's flag_complex_collapse_edges
// (include/Flag_complex_edge_collapser.h:224-482, the Boissonnat-Pritam
// collapse), the drop of every edge that is not returned (include/specseq.h:
// 410-424) and SimplexCollapse, which empties every higher simplex with a
// dropped facet (include/specseq.h:425-436, include/kernel.h:190-198).  The
// reference runs the collapse single-threaded on the host.
//
// The collapse visits the edges in filtration order.  Edge uv is dominated at
// time t when its common neighbourhood C (through the edges valid at t) is not
// empty and one w in C is adjacent to every other vertex of C.  An arriving
// edge t that is not dominated is kept (critical) and re-examines, largest id
// first, the earlier non-critical edges that close a triangle with it; each
// re-examined edge e that is no longer dominated at time e (edges valid at e:
// those before e, and the critical ones after it) is kept too and re-examines
// its own triangles.  Valid edges at the arrival of t are exactly the edges
// before t, whatever was kept, so every arrival test is independent of the
// others: one kernel runs all of them in parallel (one warp per edge).  The
// re-examinations depend on their order and run in one warp, in arrival order,
// only for the arrivals that have triangles to re-examine.  Tests are warp-
// parallel: the shorter neighbour list is intersected with the longer one
// lane by lane (binary search), and in the domination test each lane takes
// one w in C and counts its valid neighbours in C.
#include <algorithm>
#include <climits>
#include <mutex>
#include <type_traits>

#include "sspp_collapse.h"
#include "sspp_kernels.cuh"
#include "sspp_scan.cuh"

namespace sspp {

namespace {

constexpr int kWarpsA = 8;     // arrival kernel: warps per block
constexpr int kCapA = 256;     // common neighbours in shared memory per warp (arrival kernel)
constexpr int kCapB = 2048;    // common neighbours in shared memory (re-examination kernel)
constexpr int kMiscE = 0, kMiscMaxDeg = 1, kMiscCascades = 2, kMiscSteps = 3, kMiscFirst = 4;
constexpr int kOpen = 8;       // partners listed per arrival by the prefilter

unsigned grid_of(int64_t n, int threads, int64_t cap = 65536) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return unsigned(g);
}

__device__ __forceinline__ int32_t key_nbr(uint64_t k) { return int32_t(k >> 32); }
__device__ __forceinline__ int32_t key_edge(uint64_t k) { return int32_t(uint32_t(k)); }

// Per-edge flags of the re-examinations (critical, in the pending set): one
// byte per edge in global memory, or one bit per edge in shared memory when
// the edge count allows (a bit test costs a shared-memory read instead of a
// global one on the cascade's sequential path).  Only the cascade's one warp
// writes them.
struct FlagsG {
    uint8_t* p;
    __device__ __forceinline__ bool get(int32_t x) const { return p[x] != 0; }
    __device__ __forceinline__ void set(int32_t x) const { p[x] = 1; }
    __device__ __forceinline__ void clr(int32_t x) const { p[x] = 0; }
};
struct FlagsS {
    uint32_t* w;
    __device__ __forceinline__ bool get(int32_t x) const { return (w[x >> 5] >> (x & 31)) & 1u; }
    __device__ __forceinline__ void set(int32_t x) const { atomicOr(w + (x >> 5), 1u << (x & 31)); }
    __device__ __forceinline__ void clr(int32_t x) const { atomicAnd(w + (x >> 5), ~(1u << (x & 31))); }
};

// Edge x takes part in the test of edge e while edges 0..tcur have arrived:
// it precedes e, or it is critical (crit == nullptr: an arrival test, where
// only the edges before e have arrived).
template <class F>
struct ValidT {
    int32_t e, tcur;
    const F* crit;
    __device__ __forceinline__ bool operator()(int32_t x) const {
        return x < e || (crit != nullptr && x <= tcur && crit->get(x));
    }
};
using Valid = ValidT<FlagsG>;

// Common neighbours w of u and v through valid edges, ascending.  The first
// `cap` go to C (and the ids of edges uw, vw to ea, eb when given); returns
// how many there are.
template <class V>
__device__ int common_nbrs(const uint64_t* adj, const int64_t* off, int32_t u, int32_t v, const V& ok, int32_t* C,
                           int32_t* ea, int32_t* eb, int64_t cap) {
    const int lane = lane_id();
    int64_t a0 = off[u], a1 = off[u + 1], b0 = off[v], b1 = off[v + 1];
    if (a1 - a0 > b1 - b0) {  // walk the shorter list
        int64_t x = a0; a0 = b0; b0 = x;
        x = a1; a1 = b1; b1 = x;
    }
    int count = 0;
    for (int64_t base = a0; base < a1; base += 32) {
        const int64_t i = base + lane;
        bool hit = false;
        int32_t w = 0, e1 = 0, e2 = 0;
        if (i < a1) {
            const uint64_t k = adj[i];
            w = key_nbr(k);
            e1 = key_edge(k);
            if (ok(e1)) {
                const uint64_t target = uint64_t(uint32_t(w)) << 32;
                int64_t lo = b0, hi = b1;
                while (lo < hi) {
                    const int64_t mid = (lo + hi) >> 1;
                    if (adj[mid] < target) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < b1) {
                    const uint64_t k2 = adj[lo];
                    if (key_nbr(k2) == w) {
                        e2 = key_edge(k2);
                        hit = ok(e2);
                    }
                }
            }
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (hit) {
            const int p = count + __popc(m & lanemask_lt());
            if (p < cap) {
                C[p] = w;
                if (ea) {
                    ea[p] = e1;
                    eb[p] = e2;
                }
            }
        }
        count += __popc(m);
    }
    __syncwarp();
    return count;
}

// Some w in C (sorted, c >= 2) is adjacent through valid edges to every other
// vertex of C.
template <class V>
__device__ bool dominated_by_one(const uint64_t* adj, const int64_t* off, const V& ok, const int32_t* C, int c) {
    const int lane = lane_id();
    bool any = false;
    for (int base = 0; base < c && !any; base += 32) {
        const int k = base + lane;
        bool dom = false;
        if (k < c) {
            const int32_t w = C[k];
            const int64_t s0 = off[w], s1 = off[w + 1];
            if (s1 - s0 >= c - 1) {
                int cnt = 0;
                for (int64_t i = s0; i < s1; i++) {
                    const uint64_t key = adj[i];
                    if (!ok(key_edge(key))) continue;
                    const int32_t x = key_nbr(key);
                    int lo = 0, hi = c;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (C[mid] < x) lo = mid + 1;
                        else hi = mid;
                    }
                    if (lo < c && C[lo] == x) cnt++;
                }
                dom = cnt >= c - 1;
            }
        }
        any = __any_sync(kFull, dom);
    }
    return any;
}

// The same two tests for the cascade's single warp, with fewer dependent
// global loads: common_nbrs_s first copies the longer neighbour list into
// shared memory (one coalesced pass; lists longer than `slcap` take the global
// form), and dominated_by_one_s spreads the (w in C, neighbour of w) pairs over
// the lanes, so every lane loads independent entries instead of walking one
// list (C of at most 32 vertices; larger ones take the global form).
// er: the edge's neighbour-list bounds {off[u], off[u+1], off[v], off[v+1]}
template <class V>
__device__ int common_nbrs_s(const uint64_t* adj, const int64_t* off, int32_t u, int32_t v, int4 er, const V& ok,
                             int32_t* C, int32_t* ea, int32_t* eb, int64_t cap, uint64_t* sl, int slcap) {
    const int lane = lane_id();
    int64_t a0 = er.x, a1 = er.y, b0 = er.z, b1 = er.w;
    if (a1 - a0 > b1 - b0) {  // walk the shorter list
        int64_t x = a0; a0 = b0; b0 = x;
        x = a1; a1 = b1; b1 = x;
    }
    const int nb = int(b1 - b0);
    if (b1 - b0 > slcap) return common_nbrs(adj, off, u, v, ok, C, ea, eb, cap);
    for (int i = lane; i < nb; i += 32) sl[i] = adj[b0 + i];
    __syncwarp();
    int count = 0;
    for (int64_t base = a0; base < a1; base += 32) {
        const int64_t i = base + lane;
        bool hit = false;
        int32_t w = 0, e1 = 0, e2 = 0;
        if (i < a1) {
            const uint64_t k = adj[i];
            w = key_nbr(k);
            e1 = key_edge(k);
            if (ok(e1)) {
                const uint64_t target = uint64_t(uint32_t(w)) << 32;
                int lo = 0, hi = nb;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (sl[mid] < target) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < nb) {
                    const uint64_t k2 = sl[lo];
                    if (key_nbr(k2) == w) {
                        e2 = key_edge(k2);
                        hit = ok(e2);
                    }
                }
            }
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (hit) {
            const int p = count + __popc(m & lanemask_lt());
            if (p < cap) {
                C[p] = w;
                if (ea) {
                    ea[p] = e1;
                    eb[p] = e2;
                }
            }
        }
        count += __popc(m);
    }
    __syncwarp();  // sl is rewritten by the next call
    return count;
}

template <class V>
__device__ bool dominated_by_one_s(const uint64_t* adj, const int64_t* off, const int2* vrec, const V& ok,
                                   const int32_t* C, int c, int32_t* spre, int64_t* sbase, int32_t* scnt) {
    if (c > 32) return dominated_by_one(adj, off, ok, C, c);
    const int lane = lane_id();
    int deg = 0;
    if (lane < c) {
        const int2 b = vrec[C[lane]];
        const int64_t s0 = b.x, s1 = b.y;
        deg = s1 - s0 >= c - 1 ? int(s1 - s0) : 0;  // fewer neighbours than c - 1: cannot dominate
        sbase[lane] = s0;
        scnt[lane] = 0;
    }
    const int inc = warp_inclusive_scan(deg);
    const int tot = __shfl_sync(kFull, inc, 31);
    spre[lane] = inc - deg;
    __syncwarp();
    for (int base = 0; base < tot; base += 32) {
        const int p = base + lane;
        if (p < tot) {
            int lo = 0, hi = c - 1;  // the last k with spre[k] <= p
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (spre[mid] <= p) lo = mid;
                else hi = mid - 1;
            }
            const uint64_t key = adj[sbase[lo] + (p - spre[lo])];
            if (ok(key_edge(key))) {
                const int32_t x = key_nbr(key);
                int a = 0, b = c;
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    if (C[mid] < x) a = mid + 1;
                    else b = mid;
                }
                if (a < c && C[a] == x) atomicAdd(scnt + lo, 1);
            }
        }
    }
    __syncwarp();
    const bool dom = lane < c && scnt[lane] >= c - 1;
    const bool any = __any_sync(kFull, dom);
    __syncwarp();  // the scratch is rewritten by the next call
    return any;
}

// per edge and per vertex: neighbour-list bounds (int32: 2E < 2^31)
__global__ void k_cbounds(const int32_t* misc, int64_t nv, const int32_t* eu, const int32_t* ev, const int64_t* off,
                          int4* erec, int2* vrec) {
    const int64_t E = misc[kMiscE];
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < E; e += stride) {
        const int32_t u = eu[e], v = ev[e];
        erec[e] = make_int4(int32_t(off[u]), int32_t(off[u + 1]), int32_t(off[v]), int32_t(off[v + 1]));
    }
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < nv; w += stride)
        vrec[w] = make_int2(int32_t(off[w]), int32_t(off[w + 1]));
}

__global__ void k_cdeg(const int32_t* misc, const int32_t* eu, const int32_t* ev, int32_t* deg) {
    const int64_t E = misc[kMiscE];
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < E; e += int64_t(gridDim.x) * blockDim.x) {
        atomicAdd(deg + eu[e], 1);
        atomicAdd(deg + ev[e], 1);
    }
}

__global__ void k_cfill(const int32_t* misc, const int32_t* eu, const int32_t* ev, const int64_t* off, int32_t* cur,
                        uint64_t* adj) {
    const int64_t E = misc[kMiscE];
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < E; e += int64_t(gridDim.x) * blockDim.x) {
        const int32_t u = eu[e], v = ev[e];
        adj[off[u] + atomicAdd(cur + u, 1)] = (uint64_t(uint32_t(v)) << 32) | uint32_t(e);
        adj[off[v] + atomicAdd(cur + v, 1)] = (uint64_t(uint32_t(u)) << 32) | uint32_t(e);
    }
}

__device__ void heap_sort_u64(uint64_t* a, int64_t n) {
    auto sift = [&](int64_t root, int64_t end) {
        while (2 * root + 1 < end) {
            int64_t c = 2 * root + 1;
            if (c + 1 < end && a[c] < a[c + 1]) c++;
            if (a[root] >= a[c]) return;
            const uint64_t t = a[root];
            a[root] = a[c];
            a[c] = t;
            root = c;
        }
    };
    for (int64_t s = n / 2 - 1; s >= 0; s--) sift(s, n);
    for (int64_t e = n - 1; e > 0; e--) {
        const uint64_t t = a[0];
        a[0] = a[e];
        a[e] = t;
        sift(0, e);
    }
}

// sorts every neighbour list; misc[kMiscMaxDeg] = largest degree
__global__ void k_csort(int64_t nv, const int64_t* off, uint64_t* adj, int32_t* misc) {
    int32_t mx = 0;
    for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
        uint64_t* a = adj + off[v];
        const int64_t n = off[v + 1] - off[v];
        mx = n > mx ? int32_t(n) : mx;
        if (n <= 32) {
            for (int64_t i = 1; i < n; i++) {
                const uint64_t x = a[i];
                int64_t j = i - 1;
                while (j >= 0 && a[j] > x) {
                    a[j + 1] = a[j];
                    j--;
                }
                a[j + 1] = x;
            }
        } else {
            heap_sort_u64(a, n);
        }
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(misc + kMiscMaxDeg, mx);
}

// arrival test of every edge: arr 0 = dominated, 1 = kept, 2 = kept with
// triangles to re-examine
__global__ void __launch_bounds__(kWarpsA * 32) k_arrival(const int32_t* misc, const int32_t* eu, const int32_t* ev,
                                                         const uint64_t* adj, const int64_t* off, uint8_t* arr,
                                                         uint8_t* crit, int32_t* cbuf, int64_t cbuf_per_warp) {
    __shared__ int32_t sC[kWarpsA][kCapA];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gw = int64_t(blockIdx.x) * kWarpsA + w, nw = int64_t(gridDim.x) * kWarpsA;
    const int64_t E = misc[kMiscE];
    for (int64_t t = gw; t < E; t += nw) {
        const Valid ok{int32_t(t), int32_t(t), nullptr};
        const int c = common_nbrs(adj, off, eu[t], ev[t], ok, sC[w], nullptr, nullptr, kCapA);
        uint8_t r;
        if (c == 0) {
            r = 1;
        } else if (c == 1) {
            r = 0;
        } else {
            const int32_t* C = sC[w];
            if (c > kCapA) {
                int32_t* g = cbuf + gw * cbuf_per_warp;
                common_nbrs(adj, off, eu[t], ev[t], ok, g, nullptr, nullptr, cbuf_per_warp);
                C = g;
            }
            r = dominated_by_one(adj, off, ok, C, c) ? 0 : 2;
        }
        if (lane == 0) {
            arr[t] = r;
            crit[t] = r != 0;
        }
        __syncwarp();
    }
}

// An arrival re-examines only earlier edges that are not critical, and an edge
// is critical from its arrival on if it was kept then (criticality only ever
// grows).  So an arrival whose triangles' other edges were all kept at their
// own arrival pushes nothing and re-examines nothing: it leaves the cascade
// list (arr 2 -> 1).  Arrivals whose common neighbourhood does not fit in
// shared memory stay in it.  Concurrent writes only turn 2 into 1, which the
// test (arr == 0) does not see.
// The partners that can be pushed at all (at most kOpen of them) are listed
// for the cascade, which then does not recompute the arrival's triangles.
__global__ void __launch_bounds__(kWarpsA * 32) k_prefilter(const int32_t* misc, const int32_t* eu, const int32_t* ev,
                                                           const uint64_t* adj, const int64_t* off, uint8_t* arr,
                                                           int32_t* open, int8_t* nopen) {
    __shared__ int32_t sC[kWarpsA][kCapA], sA[kWarpsA][kCapA], sB[kWarpsA][kCapA];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gw = int64_t(blockIdx.x) * kWarpsA + w, nw = int64_t(gridDim.x) * kWarpsA;
    const int64_t E = misc[kMiscE];
    for (int64_t t = gw; t < E; t += nw) {
        if (arr[t] != 2) continue;
        const Valid ok{int32_t(t), int32_t(t), nullptr};
        const int c = common_nbrs(adj, off, eu[t], ev[t], ok, sC[w], sA[w], sB[w], kCapA);
        if (c > kCapA) {
            if (lane == 0) nopen[t] = -1;
            continue;
        }
        int cnt = 0;
        for (int base = 0; base < 2 * c; base += 32) {
            const int k = base + lane;
            int32_t x = -1;
            bool o = false;
            if (k < 2 * c) {
                x = k < c ? sA[w][k] : sB[w][k - c];
                o = arr[x] == 0;
            }
            const unsigned bm = __ballot_sync(kFull, o);
            const int p = cnt + __popc(bm & lanemask_lt());
            if (o && p < kOpen) open[t * kOpen + p] = x;
            cnt += __popc(bm);
        }
        if (lane == 0) {
            if (cnt == 0) arr[t] = 1;
            nopen[t] = int8_t(cnt <= kOpen ? cnt : -1);
        }
        __syncwarp();
    }
}

// max-heap of edge ids (one thread)
__device__ void heap_push(int32_t* h, int& size, int32_t x) {
    int i = size++;
    h[i] = x;
    while (i > 0) {
        const int p = (i - 1) >> 1;
        if (h[p] >= h[i]) break;
        const int32_t t = h[p];
        h[p] = h[i];
        h[i] = t;
        i = p;
    }
}

__device__ int32_t heap_pop(int32_t* h, int& size) {
    const int32_t top = h[0];
    const int32_t last = h[--size];
    int i = 0;
    for (;;) {
        int c = 2 * i + 1;
        if (c >= size) break;
        if (c + 1 < size && h[c + 1] > h[c]) c++;
        if (h[c] <= last) break;
        h[i] = h[c];
        i = c;
    }
    if (size > 0) h[i] = last;
    return top;
}

// The pending set: a max-heap of edge ids, kept by lane 0 in shared memory
// until it would overflow, then (for the rest of the launch) in global memory.
constexpr int kHeapS = 4096;

struct Pending {
    int32_t* h;
    int cap;
    int size;
    int32_t* global;  // room for every edge
};

__device__ __forceinline__ void pending_push(Pending& P, int32_t x) {
    if (P.size == P.cap && P.h != P.global) {
        for (int i = 0; i < P.size; i++) P.global[i] = P.h[i];
        P.h = P.global;
        P.cap = INT_MAX;
    }
    heap_push(P.h, P.size, x);
}

// The earlier non-critical edges uw, vw of the triangles of edge th go into
// the set: the lanes test them (no edge appears twice: uw != vw' for common
// neighbours w, w' of u and v), then lane 0 pushes the ones taken, from
// `list` (kCapB entries of shared memory; larger lists are pushed by lane 0
// directly).
template <class F>
__device__ void push_partners(const int32_t* A, const int32_t* B, int c, int32_t th, const F& crit, const F& ins,
                              int32_t* list, Pending& P) {
    const int lane = lane_id();
    if (2 * c > kCapB) {
        if (lane == 0) {
            for (int k = 0; k < c; k++) {
                const int32_t ab[2] = {A[k], B[k]};
                for (int q = 0; q < 2; q++) {
                    const int32_t x = ab[q];
                    if (x < th && !crit.get(x) && !ins.get(x)) {
                        ins.set(x);
                        pending_push(P, x);
                    }
                }
            }
        }
        __syncwarp();
        return;
    }
    int m = 0;
    for (int base = 0; base < 2 * c; base += 32) {
        const int k = base + lane;
        int32_t x = -1;
        bool want = false;
        if (k < 2 * c) {
            x = k < c ? A[k] : B[k - c];
            want = x < th && !crit.get(x) && !ins.get(x);
        }
        const unsigned bm = __ballot_sync(kFull, want);
        if (want) {
            list[m + __popc(bm & lanemask_lt())] = x;
            ins.set(x);
        }
        m += __popc(bm);
    }
    __syncwarp();
    if (lane == 0)
        for (int j = 0; j < m; j++) pending_push(P, list[j]);
    __syncwarp();
}

// Speculative cascades.  Every arrival's re-examinations run at once, one warp
// per arrival, as if no earlier arrival's cascade had kept anything: an edge
// counts as critical when the arrival pass kept it (crit_g) or this cascade
// did.  Each run records the edges it keeps and every vertex whose neighbour
// list it read (the arrival's endpoints, each popped edge's endpoints, the
// common neighbours whose lists the domination test read).  A flag this run
// read belongs to an edge in one of those lists, so an edge that an earlier
// cascade keeps can change the run only if one of its endpoints is among the
// recorded vertices; the ordered pass (k_cascade) applies a record whose
// vertices no earlier cascade touched and re-runs the others.  A run that
// outgrows its buffers records status 1 (re-run).
constexpr int kSpecWarps = 4;
constexpr int kSpecHeap = 64;
constexpr int kSpecCrit = 16;
constexpr int kSpecScan = 64;
constexpr int kSpecCap = 128;    // common neighbours per warp
constexpr int kSpecList = 256;   // staged neighbour-list entries per warp
// record: status, kept count, vertex count, 0, kept edges, their endpoints, vertices
constexpr int kRecKept = 4, kRecKA = kRecKept + kSpecCrit, kRecKB = kRecKA + kSpecCrit, kRecScan = kRecKB + kSpecCrit;
constexpr int kSpecRec = kRecScan + kSpecScan;
constexpr int kSpecMaxArrivals = 1 << 18;  // records kept; later arrivals run in order

// critical: kept by the arrival pass, or by this speculative cascade
struct FlagsSpec {
    const uint8_t* base;
    const int32_t* loc;
    const int* nloc;
    __device__ __forceinline__ bool get(int32_t x) const {
        if (base[x]) return true;
        const int n = *nloc;
        for (int i = 0; i < n; i++)
            if (loc[i] == x) return true;
        return false;
    }
};

struct SpecWarp {
    int32_t heap[kSpecHeap];
    int32_t lcrit[kSpecCrit], lca[kSpecCrit], lcb[kSpecCrit];  // kept edges and their endpoints
    int32_t scan[kSpecScan];
    int32_t C[kSpecCap], A[kSpecCap], B[kSpecCap];
    uint64_t list[kSpecList];
    int64_t sbase[32];
    int32_t spre[32], scnt[32];
    int nheap, nlcrit, nscan, abort;
};

__device__ __forceinline__ bool spec_in_heap(const SpecWarp& W, int32_t x) {
    for (int i = 0; i < W.nheap; i++)
        if (W.heap[i] == x) return true;
    return false;
}

// lane 0: add vertex x to the recorded set
__device__ __forceinline__ void spec_scan_add(SpecWarp& W, int32_t x) {
    for (int i = 0; i < W.nscan; i++)
        if (W.scan[i] == x) return;
    if (W.nscan == kSpecScan) {
        W.abort = 1;
        return;
    }
    W.scan[W.nscan++] = x;
}

// the lanes' candidates x (want) go into the pending heap, lane order
__device__ __forceinline__ void spec_push(SpecWarp& W, bool want, int32_t x) {
    const int lane = lane_id();
    const unsigned bm = __ballot_sync(kFull, want);
    for (unsigned m = bm; m; m &= m - 1) {
        const int src = __ffs(m) - 1;
        const int32_t y = __shfl_sync(kFull, x, src);
        if (lane == 0) {
            if (W.nheap == kSpecHeap) W.abort = 1;
            else heap_push(W.heap, W.nheap, y);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kSpecWarps * 32) k_cascade_spec(const int32_t* cas, const int32_t* misc,
                                                                   const int32_t* eu, const int32_t* ev,
                                                                   const uint64_t* adj, const int64_t* off,
                                                                   const uint8_t* crit_g, const int32_t* open,
                                                                   const int8_t* nopen, const int4* erec,
                                                                   const int2* vrec, int32_t* rec, int spec_cap) {
    __shared__ SpecWarp sw[kSpecWarps];
    const int lane = lane_id();
    SpecWarp& W = sw[threadIdx.x >> 5];
    const int ncas = min(misc[kMiscCascades], spec_cap);
    const FlagsSpec crit{crit_g, W.lcrit, &W.nlcrit};
    for (int i = blockIdx.x * kSpecWarps + (threadIdx.x >> 5); i < ncas; i += gridDim.x * kSpecWarps) {
        const int32_t t = cas[i];
        const int32_t u = eu[t], v = ev[t];
        const int no = nopen[t];
        if (lane == 0) {
            W.nheap = W.nlcrit = W.nscan = W.abort = 0;
            spec_scan_add(W, u);
            spec_scan_add(W, v);
        }
        __syncwarp();
        if (no >= 0) {  // the prefilter's list: edges before t, dominated at their own arrival
            const int32_t x = lane < no ? open[int64_t(t) * kOpen + lane] : -1;
            const bool want = lane < no && !crit.get(x) && !spec_in_heap(W, x);
            spec_push(W, want, x);
        } else {
            const ValidT<FlagsSpec> ok{t, t, nullptr};
            const int c = common_nbrs(adj, off, u, v, ok, W.C, W.A, W.B, kSpecCap);
            if (c > kSpecCap) {
                if (lane == 0) W.abort = 1;
            } else {
                for (int base = 0; base < 2 * c; base += 32) {
                    const int k = base + lane;
                    const int32_t x = k < 2 * c ? (k < c ? W.A[k] : W.B[k - c]) : -1;
                    const bool want = k < 2 * c && x < t && !crit.get(x) && !spec_in_heap(W, x);
                    spec_push(W, want, x);
                }
            }
        }
        __syncwarp();
        while (__shfl_sync(kFull, W.nheap > 0 && !W.abort ? 1 : 0, 0)) {
            int32_t e = 0;
            if (lane == 0) e = heap_pop(W.heap, W.nheap);
            e = __shfl_sync(kFull, e, 0);
            const int32_t a = eu[e], b = ev[e];
            if (lane == 0) {
                spec_scan_add(W, a);
                spec_scan_add(W, b);
            }
            __syncwarp();
            if (crit.get(e)) continue;
            const ValidT<FlagsSpec> ok{e, t, &crit};
            const int c = common_nbrs_s(adj, off, a, b, erec[e], ok, W.C, W.A, W.B, kSpecCap, W.list, kSpecList);
            if (c > kSpecCap) {
                if (lane == 0) W.abort = 1;
                __syncwarp();
                break;
            }
            const bool dom =
                (c == 1) || (c >= 2 && dominated_by_one_s(adj, off, vrec, ok, W.C, c, W.spre, W.sbase, W.scnt));
            if (c >= 2 && lane == 0)
                for (int k = 0; k < c; k++) spec_scan_add(W, W.C[k]);
            __syncwarp();
            if (dom) continue;
            if (lane == 0) {
                if (W.nlcrit == kSpecCrit) {
                    W.abort = 1;
                } else {
                    W.lca[W.nlcrit] = a;
                    W.lcb[W.nlcrit] = b;
                    W.lcrit[W.nlcrit++] = e;
                }
            }
            __syncwarp();
            for (int base = 0; base < 2 * c; base += 32) {
                const int k = base + lane;
                const int32_t x = k < 2 * c ? (k < c ? W.A[k] : W.B[k - c]) : -1;
                const bool want = k < 2 * c && x < e && !crit.get(x) && !spec_in_heap(W, x);
                spec_push(W, want, x);
            }
        }
        __syncwarp();
        int32_t* r = rec + int64_t(i) * kSpecRec;
        if (lane == 0) {
            r[0] = W.abort;
            r[1] = W.nlcrit;
            r[2] = W.nscan;
            r[3] = 0;
        }
        if (lane < W.nlcrit) {
            r[kRecKept + lane] = W.lcrit[lane];
            r[kRecKA + lane] = W.lca[lane];
            r[kRecKB + lane] = W.lcb[lane];
        }
        for (int k = lane; k < W.nscan; k += 32) r[kRecScan + k] = W.scan[k];
        __syncwarp();  // the warp's buffers are rewritten by its next arrival
    }
}

// Which speculative runs are exact, in parallel: if every record before i is
// exact, the edges those cascades keep are their recorded ones, so record i is
// exact when it completed and none of its vertices is an endpoint of an edge
// kept by a record before it (first_mark: the smallest record index keeping an
// edge at each vertex).  misc[kMiscFirst] gets the first record that is not
// exact (the ordered pass starts there); every record before it is applied at
// once.
__global__ void k_spec_marks(int32_t* misc, const int32_t* rec, int spec_cap, int32_t* first_mark) {
    const int n = min(misc[kMiscCascades], spec_cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) misc[kMiscFirst] = n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t* r = rec + int64_t(i) * kSpecRec;
        if (r[0] != 0) continue;
        for (int k = 0; k < r[1]; k++) {
            atomicMin(first_mark + r[kRecKA + k], i);
            atomicMin(first_mark + r[kRecKB + k], i);
        }
    }
}

__global__ void k_spec_first(int32_t* misc, const int32_t* rec, int spec_cap, const int32_t* first_mark) {
    const int n = min(misc[kMiscCascades], spec_cap);
    const int lane = lane_id();
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        const int32_t* r = rec + int64_t(i) * kSpecRec;
        bool bad = r[0] != 0;
        const int ns = r[2];
        for (int k = lane; k < ns && !bad; k += 32) bad = first_mark[r[kRecScan + k]] < i;
        if (__any_sync(kFull, bad) && lane == 0) atomicMin(misc + kMiscFirst, i);
    }
}

// also the ordered pass's starting vertex bitset: the vertices of the edges
// the applied records keep (first_mark below the first inexact record)
__global__ void k_spec_apply(const int32_t* misc, const int32_t* rec, uint8_t* crit_g, const int32_t* first_mark,
                             int64_t nv, uint32_t* dirty_words) {
    const int n = misc[kMiscFirst];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t* r = rec + int64_t(i) * kSpecRec;
        for (int k = 0; k < r[1]; k++) crit_g[r[kRecKept + k]] = 1;
    }
    const int lane = lane_id();
    const int64_t nwords = (nv + 31) >> 5;
    for (int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; w < nwords;
         w += (int64_t(gridDim.x) * blockDim.x) >> 5) {
        const int64_t v = 32 * w + lane;
        const unsigned bits = __ballot_sync(kFull, v < nv && first_mark[v] < n);
        if (lane == 0) dirty_words[w] = bits;
    }
}

// Arrivals of the cascade list read ahead per round of one warp: the arrival,
// its listed partner count and its partners.
constexpr int kAhead = 32;
constexpr int kListS = 512;  // neighbour-list entries the cascade stages in shared memory

// Re-examinations, in arrival order, by one warp (warp 0; with flags in shared
// memory the block's other warps only help load the critical flags and exit).
// The flags live in F (FlagsS: bitsets in dynamic shared memory, crit words
// then pending words; FlagsG: the global byte arrays).  An edge the cascade
// keeps is also marked in the global byte array, which k_drop_edges reads.
template <class F>
__global__ void __launch_bounds__(256) k_cascade(const int32_t* cas, int32_t* misc, const int32_t* eu,
                                                  const int32_t* ev, const uint64_t* adj, const int64_t* off,
                                                  uint8_t* crit_g, uint8_t* ins_g, int32_t* heap, const int32_t* open,
                                                  const int8_t* nopen, const int4* erec, const int2* vrec, int32_t* gC,
                                                  int32_t* gA, int32_t* gB, int64_t gcap, long long max_steps,
                                                  int* err, const int32_t* spec, int spec_cap, int64_t nv,
                                                  const uint32_t* dirty_words) {
    extern __shared__ uint32_t sbits[];
    __shared__ int32_t sC[kCapB], sA[kCapB], sB[kCapB];
    __shared__ int32_t sheap[kHeapS];
    __shared__ int32_t s_t[kAhead], s_no[kAhead], s_st[kAhead], s_nk[kAhead], s_ns[kAhead];
    __shared__ int32_t s_open[kAhead][kOpen];
    __shared__ uint64_t s_list[kListS];
    __shared__ int64_t s_base[32];
    __shared__ int32_t s_pre[32], s_cnt[32];
    const int lane = lane_id();
    const int64_t E = misc[kMiscE];
    // with spec, the arrivals before misc[kMiscFirst] were applied in parallel
    const int start = spec ? misc[kMiscFirst] : 0;
    if (start >= misc[kMiscCascades]) {
        if (threadIdx.x == 0) misc[kMiscSteps] = 0;
        return;
    }
    F crit, ins;
    FlagsS dirty{nullptr};  // with spec: vertices of edges an earlier cascade kept
    if constexpr (std::is_same<F, FlagsS>::value) {
        const int64_t nw = (E + 31) >> 5;
        crit.w = sbits;
        ins.w = sbits + nw;
        if (spec) {  // vertices of the edges the applied cascades kept (built by k_spec_apply)
            dirty.w = sbits + 2 * nw;
            for (int64_t k = threadIdx.x; k < ((nv + 31) >> 5); k += blockDim.x) dirty.w[k] = dirty_words[k];
        }
        for (int64_t k = threadIdx.x; k < nw; k += blockDim.x) {
            uint32_t word = 0;
            const int64_t e0 = 32 * k;
            if (e0 + 32 <= E) {
                const uint4* q = reinterpret_cast<const uint4*>(crit_g + e0);
                const uint4 lo = q[0], hi = q[1];
                const uint32_t parts[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
                for (int b = 0; b < 32; b++) word |= ((parts[b >> 2] >> (8 * (b & 3))) & 0xffu ? 1u : 0u) << b;
            } else {
                for (int64_t e = e0; e < E; e++) word |= (crit_g[e] ? 1u : 0u) << (e - e0);
            }
            sbits[k] = word;
            sbits[nw + k] = 0;
        }
        __syncthreads();
    } else {
        crit.p = crit_g;
        ins.p = ins_g;
    }
    if (threadIdx.x >= 32) return;
    const int ncas = misc[kMiscCascades];
    Pending P{sheap, kHeapS, 0, heap};  // kept by lane 0
    int size = 0;                        // P.size, broadcast
    long long steps = 0;
    bool fail = false;
    bool kept_any = start > 0;  // warp-uniform: some cascade may have kept an edge (dirty may be set)
    for (int i0 = start; i0 < ncas && !fail; i0 += kAhead) {
        const int nb = ncas - i0 < kAhead ? ncas - i0 : kAhead;
        if (lane < nb) {  // read ahead: nothing here changes while the cascade runs
            const int32_t t = cas[i0 + lane];
            const int no = nopen[t];
            s_t[lane] = t;
            s_no[lane] = no;
            if (spec && i0 + lane < spec_cap) {
                const int32_t* r = spec + int64_t(i0 + lane) * kSpecRec;
                s_st[lane] = r[0];
                s_nk[lane] = r[1];
                s_ns[lane] = r[2];
            } else {
                s_st[lane] = 1;
            }
            if (no > 0) {
                const int4* q = reinterpret_cast<const int4*>(open + int64_t(t) * kOpen);
                const int4 a = q[0], b = q[1];
                s_open[lane][0] = a.x; s_open[lane][1] = a.y; s_open[lane][2] = a.z; s_open[lane][3] = a.w;
                s_open[lane][4] = b.x; s_open[lane][5] = b.y; s_open[lane][6] = b.z; s_open[lane][7] = b.w;
            }
        }
        __syncwarp();
        // a record's vertices and kept edges (one or two per lane), loaded one
        // arrival ahead so that the check does not wait for them
        int32_t n_s0 = -1, n_s1 = -1, n_k = -1, n_a = -1, n_b = -1;
        auto fetch = [&](int jj) {
            n_s0 = n_s1 = n_k = n_a = n_b = -1;
            if (spec && jj < nb && s_st[jj] == 0) {
                const int32_t* r = spec + int64_t(i0 + jj) * kSpecRec;
                const int ns = s_ns[jj], nk = s_nk[jj];
                if (lane < ns) n_s0 = r[kRecScan + lane];
                if (lane + 32 < ns) n_s1 = r[kRecScan + 32 + lane];
                if (lane < nk) {
                    n_k = r[kRecKept + lane];
                    n_a = r[kRecKA + lane];
                    n_b = r[kRecKB + lane];
                }
            }
        };
        fetch(0);
        for (int j = 0; j < nb && !fail; j++) {
            const int32_t t = s_t[j];
            const int no = s_no[j];
            const int32_t c_s0 = n_s0, c_s1 = n_s1, c_k = n_k, c_a = n_a, c_b = n_b;
            fetch(j + 1);
            if (spec && s_st[j] == 0) {
                // the speculative run of this arrival stands when none of the
                // vertices it read is an endpoint of an edge an earlier cascade kept
                const bool touched =
                    kept_any && ((c_s0 >= 0 && dirty.get(c_s0)) || (c_s1 >= 0 && dirty.get(c_s1)));
                if (!__any_sync(kFull, touched)) {
                    if (c_k >= 0) {
                        crit.set(c_k);
                        crit_g[c_k] = 1;
                        dirty.set(c_a);
                        dirty.set(c_b);
                    }
                    kept_any = kept_any || s_nk[j] > 0;
                    __syncwarp();
                    continue;
                }
            }
            if (no >= 0) {  // the prefilter's list: edges before t, dominated at their own arrival
                const int32_t x = lane < no ? s_open[j][lane] : -1;
                const bool want = lane < no && !crit.get(x) && !ins.get(x);
                const unsigned bm = __ballot_sync(kFull, want);
                if (!bm) continue;  // nothing pushed, and the set is empty between arrivals
                if (want) {
                    sC[__popc(bm & lanemask_lt())] = x;
                    ins.set(x);
                }
                __syncwarp();
                if (lane == 0)
                    for (int q = 0; q < __popc(bm); q++) pending_push(P, sC[q]);
                __syncwarp();
                size = __shfl_sync(kFull, P.size, 0);
            } else {
                const ValidT<F> ok{t, t, nullptr};
                int c = common_nbrs(adj, off, eu[t], ev[t], ok, sC, sA, sB, kCapB);
                const int32_t *A = sA, *B = sB;
                if (c > kCapB) {
                    common_nbrs(adj, off, eu[t], ev[t], ok, gC, gA, gB, gcap);
                    A = gA;
                    B = gB;
                }
                push_partners(A, B, c, t, crit, ins, sC, P);
                size = __shfl_sync(kFull, P.size, 0);
            }
            while (size > 0) {
                if (++steps > max_steps) {
                    fail = true;
                    break;
                }
                int32_t e = 0;
                if (lane == 0) {
                    e = heap_pop(P.h, P.size);
                    ins.clr(e);
                    // the next pop is usually the current top: start fetching its bounds
                    if (P.size > 0) asm volatile("prefetch.global.L1 [%0];" ::"l"(erec + P.h[0]));
                }
                e = __shfl_sync(kFull, e, 0);
                size = __shfl_sync(kFull, P.size, 0);
                __syncwarp();
                if (crit.get(e)) continue;
                const ValidT<F> ok{e, t, &crit};
                const int4 er = erec[e];  // both endpoints' list bounds in one load
                int c = common_nbrs_s(adj, off, eu[e], ev[e], er, ok, sC, sA, sB, kCapB, s_list, kListS);
                const int32_t *C = sC, *A = sA, *B = sB;
                if (c > kCapB) {
                    common_nbrs(adj, off, eu[e], ev[e], ok, gC, gA, gB, gcap);
                    C = gC;
                    A = gA;
                    B = gB;
                }
                const bool dom = (c == 1) || (c >= 2 && dominated_by_one_s(adj, off, vrec, ok, C, c, s_pre, s_base, s_cnt));
                if (dom) continue;
                if (lane == 0) {
                    crit.set(e);
                    crit_g[e] = 1;
                    if (spec) {
                        dirty.set(eu[e]);
                        dirty.set(ev[e]);
                    }
                }
                kept_any = true;
                __syncwarp();
                push_partners(A, B, c, e, crit, ins, sC, P);
                size = __shfl_sync(kFull, P.size, 0);
            }
        }
        __syncwarp();  // s_t / s_no / s_open are rewritten by the next round
    }
    if (lane == 0) {
        misc[kMiscSteps] = int32_t(steps > INT_MAX ? INT_MAX : steps);
        if (fail) atomicOr(err, ERRB_TIMEOUT);
    }
}

__global__ void k_drop_edges(const int32_t* misc, const uint8_t* crit, const int32_t* ecol, uint8_t* dropped) {
    const int64_t E = misc[kMiscE];
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < E; e += int64_t(gridDim.x) * blockDim.x)
        if (!crit[e]) dropped[ecol[e]] = 1;
}

// a simplex of dimension >= 2 with a dropped facet is dropped
__global__ void k_drop_up(int32_t cb, int32_t ce, const int32_t* arena, const uint64_t* desc, uint8_t* dropped) {
    for (int64_t j = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < ce; j += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t d = desc[j];
        const int32_t* c = arena + desc_off(d) + kHdr;
        const uint32_t len = desc_len(d);
        for (uint32_t k = 0; k < len; k++)
            if (dropped[c[k]]) {
                dropped[j] = 1;
                break;
            }
    }
}

__global__ void k_empty_dropped(int64_t n, int32_t* arena, uint64_t* desc, const uint8_t* dropped,
                                long long* counters) {
    long long cnt = 0;
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        if (!dropped[j]) continue;
        const uint64_t d = desc[j];
        desc[j] = pack_desc(desc_off(d), 0);
        arena[desc_off(d)] = 0;
        cnt++;
    }
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) cnt_add(&counters[CNT_DROPPED], cnt);
}

// Dynamic shared memory the bitset cascade may take on this device (the
// opt-in maximum less its static buffers), raised once per device.
size_t cascade_shared_limit() {
    static std::mutex mu;
    static int limit[64] = {};
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[dev]) {
        int optin = 0;
        cudaFuncAttributes fa{};
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_cascade<FlagsS>) == cudaSuccess && optin > int(fa.sharedSizeBytes)) {
            const int want = optin - int(fa.sharedSizeBytes);
            if (cudaFuncSetAttribute(k_cascade<FlagsS>, cudaFuncAttributeMaxDynamicSharedMemorySize, want) ==
                cudaSuccess)
                limit[dev] = want;
        }
        cudaGetLastError();
        done[dev] = true;
    }
    return size_t(limit[dev]);
}

// stream-ordered, like the engine's other buffers
template <typename T>
cudaError_t grow_buf(T*& p, int64_t want, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    return cudaMallocAsync(reinterpret_cast<void**>(&p), size_t(want > 0 ? want : 1) * sizeof(T), s);
}

}  // namespace

void collapse_free(CollapseScratch& S) {
    void* ptrs[] = {S.eu, S.ev, S.ecol, S.deg, S.adj_off, S.adj, S.arr, S.crit, S.ins, S.heap, S.cas, S.open, S.nopen,
                    S.cbuf, S.misc, S.erec, S.vrec, S.spec, S.first_mark, S.dirty_words};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    S = CollapseScratch();
}

int collapse(Device& D, const DimInfo& info, uint8_t* dropped, CollapseScratch& S, cudaStream_t s,
             const char** err_msg) {
    const int64_t n = D.n;
    int launches = 0;
    cudaMemsetAsync(dropped, 0, size_t(n), s);
    const int32_t eb = info.col_begin[1], ee = info.col_end[1];
    const int64_t nv = info.col_end[0] - info.col_begin[0];
    const int64_t ne = ee > eb ? ee - eb : 0;
    if (ne == 0 || nv == 0) return 0;
    *err_msg = "edge collapse: device allocation failed";
    if (ne > S.cap_e) {
        if (grow_buf(S.eu, ne, s) || grow_buf(S.ev, ne, s) || grow_buf(S.ecol, ne, s) || grow_buf(S.adj, 2 * ne, s) ||
            grow_buf(S.arr, ne, s) || grow_buf(S.crit, ne, s) || grow_buf(S.ins, ne, s) || grow_buf(S.heap, ne, s) ||
            grow_buf(S.cas, ne, s) || grow_buf(S.open, ne * kOpen, s) || grow_buf(S.nopen, ne, s) ||
            grow_buf(S.erec, ne, s))
            return -1;
        S.cap_e = ne;
    }
    if (nv + 1 > S.cap_v) {
        if (grow_buf(S.deg, nv + 1, s) || grow_buf(S.adj_off, nv + 1, s) || grow_buf(S.vrec, nv + 1, s) ||
            grow_buf(S.first_mark, nv + 1, s) || grow_buf(S.dirty_words, (nv + 32) / 32, s))
            return -1;
        S.cap_v = nv + 1;
    }
    if (!S.misc && grow_buf(S.misc, 8, s)) return -1;
    cudaMemsetAsync(S.misc, 0, 8 * sizeof(int32_t), s);
    // edge list: the 2-row columns of dimension 1, in filtration order
    {
        const uint64_t* desc = D.desc;
        const int32_t* arena = D.arena;
        int32_t* eu = S.eu;
        int32_t* ev = S.ev;
        int32_t* ecol = S.ecol;
        scan([=] __device__(int64_t i) -> int64_t { return desc_len(desc[eb + i]) == 2 ? 1 : 0; },
             [=] __device__(int64_t i, int64_t pre, int64_t v) {
                 if (v) {
                     const int32_t* c = arena + desc_off(desc[eb + i]) + kHdr;
                     eu[pre] = c[0];
                     ev[pre] = c[1];
                     ecol[pre] = int32_t(eb + i);
                 }
             },
             ne, D.blk, s);
        launches += 3;
    }
    // the edge count E for the kernels (low 32 bits of the int64 total: E <= ne < 2^30
    // is checked here); the host sizes its launches by ne and reads E below,
    // with the largest degree, in one synchronisation
    if (2 * ne >= int64_t(INT32_MAX)) {  // neighbour-list offsets are kept as int32
        *err_msg = "edge collapse: more than 2^30 edge columns";
        return -1;
    }
    cudaMemcpyAsync(S.misc + kMiscE, D.blk + scan_blocks(ne), sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    // adjacency: (neighbour, edge id), ascending per vertex
    cudaMemsetAsync(S.deg, 0, sizeof(int32_t) * (nv + 1), s);
    k_cdeg<<<grid_of(ne, 256), 256, 0, s>>>(S.misc, S.eu, S.ev, S.deg);
    {
        const int32_t* deg = S.deg;
        int64_t* off = S.adj_off;
        scan([=] __device__(int64_t v) -> int64_t { return v < nv ? deg[v] : 0; },
             [=] __device__(int64_t v, int64_t pre, int64_t) { off[v] = pre; }, nv + 1, D.blk, s);
    }
    cudaMemsetAsync(S.deg, 0, sizeof(int32_t) * (nv + 1), s);
    k_cfill<<<grid_of(ne, 256), 256, 0, s>>>(S.misc, S.eu, S.ev, S.adj_off, S.deg, S.adj);
    k_csort<<<grid_of(nv, 128), 128, 0, s>>>(nv, S.adj_off, S.adj, S.misc);
    k_cbounds<<<grid_of(std::max<int64_t>(ne, nv), 256), 256, 0, s>>>(S.misc, nv, S.eu, S.ev, S.adj_off, S.erec, S.vrec);
    launches += 7;
    int32_t mm[2] = {0, 0};  // edge count, largest degree
    cudaMemcpyAsync(mm, S.misc + kMiscE, sizeof(mm), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        *err_msg = "edge collapse: adjacency build";
        return -1;
    }
    const int64_t E = mm[0];
    const int32_t maxdeg = mm[1];
    if (E == 0) return launches;
    // overflow buffers for common neighbourhoods larger than shared memory
    int64_t warps_a = std::min<int64_t>(E, 148 * 64);
    int64_t per_warp = maxdeg > kCapA ? maxdeg : 0;
    if (per_warp > 0) warps_a = std::max<int64_t>(1, std::min<int64_t>(warps_a, (int64_t(1) << 26) / per_warp));
    warps_a = (warps_a + kWarpsA - 1) / kWarpsA * kWarpsA;  // whole blocks, each warp with its buffer
    const int64_t gcap = maxdeg > kCapB ? maxdeg : 0;
    const int64_t want = std::max<int64_t>(warps_a * per_warp, 3 * gcap) + 1;
    if (want > S.cap_cbuf) {
        if (grow_buf(S.cbuf, want, s)) return -1;
        S.cap_cbuf = want;
    }
    k_arrival<<<unsigned(warps_a / kWarpsA), kWarpsA * 32, 0, s>>>(
        S.misc, S.eu, S.ev, S.adj, S.adj_off, S.arr, S.crit, S.cbuf, per_warp);
    k_prefilter<<<unsigned(warps_a / kWarpsA), kWarpsA * 32, 0, s>>>(S.misc, S.eu, S.ev, S.adj, S.adj_off, S.arr,
                                                                      S.open, S.nopen);
    launches++;
    {
        const uint8_t* arr = S.arr;
        int32_t* cas = S.cas;
        scan([=] __device__(int64_t t) -> int64_t { return arr[t] == 2 ? 1 : 0; },
             [=] __device__(int64_t t, int64_t pre, int64_t v) {
                 if (v) cas[pre] = int32_t(t);
             },
             E, D.blk, s);
    }
    // count of arrivals with re-examinations (fits in int32: E does)
    cudaMemcpyAsync(S.misc + kMiscCascades, D.blk + scan_blocks(E), sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    // every pop either keeps an edge (at most E times) or discards one inserted
    // by a kept edge's triangles; the bound only guards against a corrupted set
    const double bound = 64.0 * double(E) * double(maxdeg + 1) + double(1 << 20);
    const long long max_steps = bound > 4.0e18 ? (long long)4e18 : (long long)bound;
    // flags as shared-memory bitsets while they fit next to the kernel's
    // static buffers, else the global byte arrays
    const size_t bits_bytes = size_t(2) * size_t((E + 31) >> 5) * sizeof(uint32_t);
    const size_t spec_bytes = bits_bytes + size_t((nv + 31) >> 5) * sizeof(uint32_t);  // plus the vertex bitset
    const size_t limit = cascade_shared_limit();
    if (bits_bytes <= limit) {
        // speculative cascades first, when the vertex bitset fits beside the edge flags
        const int spec_cap = int(std::min<int64_t>(E, kSpecMaxArrivals));
        int32_t* spec = nullptr;
        if (spec_bytes <= limit) {
            const int64_t want_rec = int64_t(spec_cap) * kSpecRec;
            if (want_rec > S.cap_spec) {
                if (grow_buf(S.spec, want_rec, s)) return -1;
                S.cap_spec = want_rec;
            }
            spec = S.spec;
            k_cascade_spec<<<grid_of(spec_cap, kSpecWarps, 148 * 16), kSpecWarps * 32, 0, s>>>(
                S.cas, S.misc, S.eu, S.ev, S.adj, S.adj_off, S.crit, S.open, S.nopen, S.erec, S.vrec, S.spec, spec_cap);
            cudaMemsetAsync(S.first_mark, 0x7f, sizeof(int32_t) * size_t(nv), s);  // 0x7f7f7f7f: no record
            k_spec_marks<<<grid_of(spec_cap, 256, 148 * 8), 256, 0, s>>>(S.misc, S.spec, spec_cap, S.first_mark);
            k_spec_first<<<grid_of(int64_t(spec_cap) * 32, 256, 148 * 16), 256, 0, s>>>(S.misc, S.spec, spec_cap,
                                                                                        S.first_mark);
            k_spec_apply<<<grid_of(std::max<int64_t>(spec_cap, (nv + 31) / 32 * 32), 256, 148 * 8), 256, 0, s>>>(
                S.misc, S.spec, S.crit, S.first_mark, nv, S.dirty_words);
            launches += 4;
        }
        k_cascade<FlagsS><<<1, 256, spec ? spec_bytes : bits_bytes, s>>>(
            S.cas, S.misc, S.eu, S.ev, S.adj, S.adj_off, S.crit, S.ins, S.heap, S.open, S.nopen, S.erec, S.vrec, S.cbuf,
            S.cbuf + gcap, S.cbuf + 2 * gcap, gcap, max_steps, D.err, spec, spec_cap, nv, S.dirty_words);
    } else {
        cudaMemsetAsync(S.ins, 0, size_t(E), s);
        k_cascade<FlagsG><<<1, 32, 0, s>>>(S.cas, S.misc, S.eu, S.ev, S.adj, S.adj_off, S.crit, S.ins, S.heap,
                                           S.open, S.nopen, S.erec, S.vrec, S.cbuf, S.cbuf + gcap, S.cbuf + 2 * gcap,
                                           gcap, max_steps, D.err, nullptr, 0, nv, nullptr);
    }
    k_drop_edges<<<grid_of(E, 256), 256, 0, s>>>(S.misc, S.crit, S.ecol, dropped);
    launches += 7;
    for (int d = 2; d <= kMaxDim; d++) {
        const int32_t cb = info.col_begin[d], ce = info.col_end[d];
        if (ce <= cb) continue;
        k_drop_up<<<grid_of(ce - cb, 256), 256, 0, s>>>(cb, ce, D.arena, D.desc, dropped);
        launches++;
    }
    k_empty_dropped<<<grid_of(n, 256), 256, 0, s>>>(n, D.arena, D.desc, dropped, D.counters);
    launches++;
    *err_msg = nullptr;
    return launches;
}

}  // namespace sspp
