// High-dimension guided clearing (model bit 1).
//
// Reference counterparts: init_contain_vertics (include/kernel.h:121-188:
// vertex set of a simplex from its first two facets), maxdim_clear_init
// (include/kernel.h:202-292: the clearing test on the top dimension), the
// neighbour lists and binomial key tables (include/specseq.h:215-259) and the
// driver (include/specseq.h:523-541).
//
// Test.  For a top-dimension simplex s = (v0 < ... < vD) the candidates w are
// the neighbours of v0 in ascending order, at most max_iteration of them.  If
// w is adjacent to every vertex of s, t = s + {w} is a simplex of the flag
// complex; when every other facet of t exists and precedes s, s is the
// youngest facet of t, so the column of s is a sum of earlier columns and s is
// positive: its column is cleared.  Facets are found through an open-
// addressing hash of the top-dimension vertex tuples (the reference sorts
// combinatorial-number keys and binary-searches them).  A group of lanes
// (max_iteration rounded up to a power of two, at most a warp) handles one
// simplex, one lane one candidate.
//
// The reference walks the neighbour lists with a comparison in the wrong
// direction (include/kernel.h:217), which only ever accepts the smallest
// common neighbour; this kernel intersects the lists as intended.  Both are
// sound, so the persistence pairs are the same; more columns are cleared here.
// Only edges and simplices that survive an edge collapse take part.
#include <climits>

#include "sspp_highclear.h"
#include "sspp_kernels.cuh"
#include "sspp_scan.cuh"

namespace sspp {

static unsigned gridn(int64_t n, int t, int cap = 65536) {
    int64_t g = (n + t - 1) / t;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return unsigned(g);
}

// The vertex tuple of a d-simplex (d >= 1) from its first two facets c0, c1:
// the union of their sorted d-tuples is a sorted (d+1)-tuple; all -1 if not.
__device__ __forceinline__ void tuple_union(int d, int32_t c0, int32_t c1, int32_t fb, const int32_t* tup_f,
                                            int32_t* out) {
    int32_t a[kMaxDim + 1], b[kMaxDim + 1];
    for (int k = 0; k < d; k++) {
        a[k] = (d == 1) ? c0 : tup_f[int64_t(c0 - fb) * d + k];
        b[k] = (d == 1) ? c1 : tup_f[int64_t(c1 - fb) * d + k];
    }
    int ia = 0, ib = 0, m = 0;
    bool ok = true;
    while ((ia < d || ib < d) && m <= d) {
        int32_t x;
        if (ib >= d || (ia < d && a[ia] < b[ib])) x = a[ia++];
        else if (ia >= d || b[ib] < a[ia]) x = b[ib++];
        else { x = a[ia++]; ib++; }
        if (x < 0) ok = false;
        out[m++] = x;
    }
    if (!ok || m != d + 1 || ia != d || ib != d) {
        for (int k = 0; k <= d; k++) out[k] = -1;
    }
}

// Vertex tuple of every column of dimension d >= 1 (sorted, d+1 vertices),
// from the first two facets' tuples.  tup_d / tup_f point at the tuple arrays of
// dims d and d-1 (dim-0 tuples are the vertex indices themselves).
__global__ void k_tuples(int32_t cb, int32_t ce, int d, int32_t fb, const int32_t* arena, const uint64_t* desc,
                         const int32_t* tup_f, int32_t* tup_d, int* err) {
    for (int64_t i = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ce; i += int64_t(gridDim.x) * blockDim.x) {
        uint64_t ds = desc[i];
        const int32_t* c = arena + desc_off(ds) + kHdr;
        int32_t* out = tup_d + (i - cb) * (d + 1);
        if (desc_len(ds) < 2 || desc_len(ds) != uint32_t(d + 1)) {
            // not a simplicial boundary (edge with < 2 vertices etc.): no tuple
            for (int k = 0; k <= d; k++) out[k] = -1;
            continue;
        }
        tuple_union(d, c[0], c[1], fb, tup_f, out);
    }
}

// The same tuples read from the input matrix through the reorder's index maps
// (perm, newidx), so that they need only the dimension assignment, not the
// reordered columns: a face index outside the input, or outside dimension
// d-1, gives no tuple (the reorder reports such a matrix as malformed).
__global__ void k_tuples_in(int32_t cb, int32_t ce, int d, int32_t fb, int32_t fe, const int32_t* perm,
                            const int32_t* newidx, const int64_t* colptr, const int32_t* rows, int64_t n,
                            const int32_t* tup_f, int32_t* tup_d) {
    for (int64_t i = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ce; i += int64_t(gridDim.x) * blockDim.x) {
        int32_t* out = tup_d + (i - cb) * (d + 1);
        const int64_t j = perm[i], a = colptr[j];
        bool ok = colptr[j + 1] - a == d + 1;
        int32_t f0 = -1, f1 = -1;
        if (ok) {
            const int32_t r0 = rows[a], r1 = rows[a + 1];
            ok = r0 >= 0 && r0 < n && r1 >= 0 && r1 < n;
            if (ok) {
                f0 = newidx[r0];
                f1 = newidx[r1];
                ok = f0 >= fb && f0 < fe && f1 >= fb && f1 < fe;
            }
        }
        if (!ok) {
            for (int k = 0; k <= d; k++) out[k] = -1;
            continue;
        }
        tuple_union(d, f0, f1, fb, tup_f, out);
    }
}

__device__ __forceinline__ uint32_t tuple_hash(const int32_t* t, int k) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < k; i++) {
        h ^= uint64_t(uint32_t(t[i])) + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h *= 0xBF58476D1CE4E5B9ull;
    }
    h ^= h >> 31;
    return uint32_t(h);
}

__global__ void k_hash_insert(int32_t cb, int32_t ce, int k, const int32_t* tup, const uint8_t* dropped, int32_t* table,
                              uint32_t mask) {
    for (int64_t i = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ce; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t* t = tup + (i - cb) * k;
        if (t[0] < 0 || (dropped && dropped[i])) continue;
        uint32_t h = tuple_hash(t, k) & mask;
        for (uint32_t probe = 0; probe <= mask; probe++) {
            int32_t old = atomicCAS(table + h, -1, int32_t(i));
            if (old == -1) break;
            h = (h + 1) & mask;
        }
    }
}

// column of the top-dimension simplex with vertex tuple t, or -1
__device__ int32_t hash_find(const int32_t* t, int k, const int32_t* table, uint32_t mask, const int32_t* tup,
                             int32_t cb) {
    uint32_t h = tuple_hash(t, k) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        int32_t c = table[h];
        if (c < 0) return -1;
        const int32_t* u = tup + int64_t(c - cb) * k;
        bool eq = true;
        for (int j = 0; j < k && eq; j++) eq = (u[j] == t[j]);
        if (eq) return c;
        h = (h + 1) & mask;
    }
    return -1;
}

// adjacency of the vertices (reordered vertex index = column index in [0, V))
// (edges from their vertex tuples, tup1 = tuples of dimension 1)
__global__ void k_degree(int32_t eb, int32_t ee, const int32_t* tup1, const uint8_t* dropped, int32_t* deg) {
    for (int64_t i = eb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ee; i += int64_t(gridDim.x) * blockDim.x) {
        const int2 c = reinterpret_cast<const int2*>(tup1)[i - eb];
        if (c.x < 0 || (dropped && dropped[i])) continue;
        atomicAdd(deg + c.x, 1);
        atomicAdd(deg + c.y, 1);
    }
}

__global__ void k_adj_fill(int32_t eb, int32_t ee, const int32_t* tup1, const uint8_t* dropped, const int64_t* adj_off,
                           int32_t* fill, int32_t* adj, int32_t* src) {
    for (int64_t i = eb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ee; i += int64_t(gridDim.x) * blockDim.x) {
        const int2 c = reinterpret_cast<const int2*>(tup1)[i - eb];
        if (c.x < 0 || (dropped && dropped[i])) continue;
        const int32_t u = c.x, v = c.y;
        const int64_t pu = adj_off[u] + atomicAdd(fill + u, 1), pv = adj_off[v] + atomicAdd(fill + v, 1);
        adj[pu] = v;
        adj[pv] = u;
        if (src) {
            src[pu] = u;
            src[pv] = v;
        }
    }
}

// heap sort of one adjacency list (any length; O(d log d))
__device__ void heap_sort(int32_t* a, int64_t n) {
    auto sift = [&](int64_t root, int64_t end) {
        while (2 * root + 1 < end) {
            int64_t c = 2 * root + 1;
            if (c + 1 < end && a[c] < a[c + 1]) c++;
            if (a[root] >= a[c]) return;
            int32_t t = a[root]; a[root] = a[c]; a[c] = t;
            root = c;
        }
    };
    for (int64_t s = n / 2 - 1; s >= 0; s--) sift(s, n);
    for (int64_t e = n - 1; e > 0; e--) {
        int32_t t = a[0]; a[0] = a[e]; a[e] = t;
        sift(0, e);
    }
}

// a short list (n <= K) sorted in registers: all K loads in flight together,
// then a bitonic sorting network (every index a compile-time constant), with
// INT32_MAX padding that sorts to the end
template <int K>
__device__ __forceinline__ void sort_short(int32_t* p, int n) {
    int32_t a[K];
#pragma unroll
    for (int i = 0; i < K; i++) a[i] = i < n ? p[i] : INT32_MAX;
#pragma unroll
    for (int k = 2; k <= K; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int i = 0; i < K; i++) {
                const int l = i ^ j;
                if (l > i) {
                    const int32_t x = a[i], y = a[l];
                    const bool swap = ((i & k) == 0) ? (x > y) : (x < y);
                    a[i] = swap ? y : x;
                    a[l] = swap ? x : y;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < K; i++)
        if (i < n) p[i] = a[i];
}

__global__ void k_adj_sort(int64_t nv, const int64_t* adj_off, int32_t* adj) {
    for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
        int32_t* a = adj + adj_off[v];
        const int64_t n = adj_off[v + 1] - adj_off[v];
        if (n <= 1) continue;
        if (n <= 16) sort_short<16>(a, int(n));
        else if (n <= 32) sort_short<32>(a, int(n));
        else heap_sort(a, n);
    }
}

__device__ __forceinline__ bool adj_has(const int32_t* adj, const int64_t* adj_off, int32_t u, int32_t w) {
    int64_t lo = adj_off[u], hi = adj_off[u + 1];
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (adj[mid] < w) lo = mid + 1;
        else hi = mid;
    }
    return lo < adj_off[u + 1] && adj[lo] == w;
}

// Candidate masks.  The candidates of a simplex are the first L(a) =
// min(max_iteration, deg a) neighbours of its smallest vertex a, so whether a
// candidate is adjacent to another vertex b of the simplex depends on the edge
// (a, b) alone: entry (a, b) of the lists gets the bit mask of a's candidates
// that are neighbours of b (a merge of a's first L(a) neighbours with b's
// sorted list).  Only entries with b > a are read (a is the smallest vertex of
// the simplex), so the others get 0.  One thread per list entry; src gives
// the entry's vertex.
__global__ void k_adj_masks(int64_t nv, const int32_t* src, const int32_t* adj, const int64_t* adj_off, int max_iter,
                            uint64_t* nmask) {
    const int64_t entries = adj_off[nv];  // the lists hold the surviving edges only
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < entries; e += int64_t(gridDim.x) * blockDim.x) {
        const int32_t a = src[e], b = adj[e];
        uint64_t m = 0;
        if (b > a) {
            const int64_t a0 = adj_off[a], b0 = adj_off[b];
            const int64_t na = adj_off[a + 1] - a0, nb = adj_off[b + 1] - b0;
            const int L = int(na < max_iter ? na : max_iter);
            int q = 0;
            int64_t t = 0;
            while (q < L && t < nb) {
                const int32_t x = adj[a0 + q], y = adj[b0 + t];
                if (x == y) m |= 1ull << q;
                q += x <= y;
                t += y <= x;
            }
        }
        nmask[e] = m;
    }
}

// One thread per top-dimension simplex s = (v0 < ... < vD): the candidates
// adjacent to every vertex are the AND of the masks of the entries (v0, vj),
// found by binary search in v0's list (every edge of a surviving simplex
// survives); each such candidate w then needs every other facet of s + {w}
// to exist and precede s.
__global__ void __launch_bounds__(256) k_highclear_masks(int32_t cb, int32_t ce, int D, const int32_t* tup,
                                                         const int32_t* adj, const int64_t* adj_off,
                                                         const uint64_t* nmask, const int32_t* table, uint32_t mask,
                                                         const uint8_t* dropped, uint8_t* cleared,
                                                         long long* counters) {
    const int k = D + 1;
    long long found_total = 0;
    for (int64_t i = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ce; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t* s = tup + (i - cb) * k;
        int32_t sv[kMaxDim + 1];
#pragma unroll
        for (int j = 0; j <= kMaxDim; j++) sv[j] = j < k ? s[j] : 0;
        if (sv[0] < 0 || (dropped && dropped[i])) continue;
        const int64_t a0 = adj_off[sv[0]];
        const int n0 = int(adj_off[sv[0] + 1] - a0);
        uint64_t m = ~0ull;
#pragma unroll
        for (int j = 1; j <= kMaxDim; j++) {
            if (j < k) {
                int lo = 0, hi = n0;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (adj[a0 + mid] < sv[j]) lo = mid + 1;
                    else hi = mid;
                }
                m = (lo < n0 && adj[a0 + lo] == sv[j]) ? m & nmask[a0 + lo] : 0;
            }
        }
        bool found = false;
        while (m && !found) {
            const int q = __ffsll(static_cast<long long>(m)) - 1;
            m &= m - 1;
            const int32_t w = adj[a0 + q];
            // t = s + {w}, sorted; every facet other than s must exist and precede column i
            int32_t t[kMaxDim + 2];
            int c = 0;
            bool placed = false;
            for (int j = 0; j < k; j++) {
                if (!placed && w < sv[j]) { t[c++] = w; placed = true; }
                t[c++] = sv[j];
            }
            if (!placed) t[c++] = w;
            bool ok = true;
            int32_t f[kMaxDim + 1];
            for (int drop = 0; drop <= k && ok; drop++) {
                if (t[drop] == w) continue;  // that facet is s itself
                int mm = 0;
                for (int j = 0; j <= k; j++)
                    if (j != drop) f[mm++] = t[j];
                const int32_t col = hash_find(f, k, table, mask, tup, cb);
                ok = col >= 0 && col < i;
            }
            found = ok;
        }
        if (found) {
            cleared[i] = 1;
            found_total++;
        }
    }
    found_total = warp_sum(found_total);
    if ((threadIdx.x & 31) == 0 && found_total) cnt_add(&counters[CNT_HIGHCLEAR], found_total);
}

// G lanes per top-dimension simplex (G = max_iteration rounded up to a power
// of two, at most 32), one lane per candidate; a warp takes 32 / G simplices
// at a time, so a small max_iteration does not leave most lanes idle.  The
// candidates are read with one coalesced load per group; for each further
// vertex of the simplex the group stages that vertex's neighbour list in
// shared memory (coalesced; lists longer than kNbrCap are searched in global
// memory instead) and every surviving candidate is binary-searched there.
constexpr int kHcThreads = 256;
constexpr int kNbrCap = 64;

__device__ __forceinline__ bool sorted_has(const int32_t* a, int n, int32_t w) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < w) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && a[lo] == w;
}

template <int G>
__global__ void __launch_bounds__(kHcThreads) k_highclear(int32_t cb, int32_t ce, int D, int max_iter,
                                                          const int32_t* tup, const int32_t* adj,
                                                          const int64_t* adj_off, const int32_t* table, uint32_t mask,
                                                          const uint8_t* dropped, uint8_t* cleared,
                                                          long long* counters) {
    constexpr int kPer = 32 / G;  // simplices per warp
    constexpr unsigned kGroupMask = G == 32 ? 0xffffffffu : ((1u << G) - 1);
    __shared__ int32_t s_nbr[kHcThreads / 32][kPer][kNbrCap];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, grp = lane / G, gl = lane % G;
    const unsigned gmask = kGroupMask << (grp * G);
    int32_t* nbuf = s_nbr[wid][grp];
    const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int k = D + 1;
    long long found_total = 0;
    for (int64_t wb = cb + warp * kPer; wb < ce; wb += nwarps * kPer) {
        const int64_t i = wb + grp;
        const int32_t* s = tup + (i - cb) * k;
        const bool valid = i < ce && s[0] >= 0 && !(dropped && dropped[i]);
        const int32_t v0 = valid ? s[0] : 0;
        const int64_t a0 = valid ? adj_off[v0] : 0;
        const int64_t nb = valid ? adj_off[v0 + 1] - a0 : 0;
        const int64_t limit = nb < max_iter ? nb : max_iter;
        bool found = false;
        for (int64_t base = 0;; base += G) {
            const bool act = valid && !found && base < limit;
            if (!__any_sync(kFull, act)) break;
            const int64_t q = base + gl;
            bool ok = act && q < limit;
            const int32_t w = ok ? adj[a0 + q] : -1;
            // w must be adjacent to every other vertex of s
            for (int j = 1; j < k; j++) {
                if (!__any_sync(kFull, ok)) break;
                const bool gany = (__ballot_sync(kFull, ok) & gmask) != 0;
                const int32_t u = gany ? s[j] : 0;
                const int64_t b0 = gany ? adj_off[u] : 0;
                const int len = gany ? int(adj_off[u + 1] - b0) : 0;
                const bool staged = len <= kNbrCap;
                if (gany && staged)
                    for (int t = gl; t < len; t += G) nbuf[t] = adj[b0 + t];
                __syncwarp();
                if (ok) ok = staged ? sorted_has(nbuf, len, w) : adj_has(adj, adj_off, u, w);
                __syncwarp();  // the next vertex's list overwrites the buffer
            }
            if (ok) {
                // t = s + {w}, sorted; every facet other than s must exist and precede column i
                int32_t t[kMaxDim + 2];
                int m = 0;
                bool placed = false;
                for (int j = 0; j < k; j++) {
                    if (!placed && w < s[j]) { t[m++] = w; placed = true; }
                    t[m++] = s[j];
                }
                if (!placed) t[m++] = w;
                int32_t f[kMaxDim + 1];
                for (int drop = 0; drop <= k && ok; drop++) {
                    if (t[drop] == w) continue;  // that facet is s itself
                    int mm = 0;
                    for (int j = 0; j <= k; j++)
                        if (j != drop) f[mm++] = t[j];
                    int32_t c = hash_find(f, k, table, mask, tup, cb);
                    ok = (c >= 0 && c < i);
                }
            }
            const unsigned bl = __ballot_sync(kFull, ok);
            found = found || ((bl >> (grp * G)) & kGroupMask) != 0;
        }
        if (valid && found && gl == 0) {
            cleared[i] = 1;
            found_total++;
        }
    }
    found_total = warp_sum(found_total);
    if (lane == 0 && found_total) cnt_add(&counters[CNT_HIGHCLEAR], found_total);
}

int highclear(Device& D, const DimInfo& info, int max_iteration, const uint8_t* dropped, HighclearScratch& S,
              cudaStream_t s, bool from_input) {
    // top dimension with columns
    int top = -1;
    for (int d = kMaxDim; d >= 1; d--)
        if (info.col_end[d] > info.col_begin[d]) { top = d; break; }
    if (top < 1 || max_iteration <= 0) return 0;
    int launches = 0;
    // tuples of dims 1..top
    const int32_t* prev = nullptr;
    for (int d = 1; d <= top; d++) {
        int32_t cb = info.col_begin[d], ce = info.col_end[d];
        if (from_input)
            k_tuples_in<<<gridn(ce - cb, 256), 256, 0, s>>>(cb, ce, d, info.col_begin[d - 1], info.col_end[d - 1],
                                                           D.perm, D.newidx, D.in_colptr, D.in_rows, D.n, prev,
                                                           S.tup[d]);
        else
            k_tuples<<<gridn(ce - cb, 256), 256, 0, s>>>(cb, ce, d, info.col_begin[d - 1], D.arena, D.desc, prev,
                                                        S.tup[d], D.err);
        launches++;
        prev = S.tup[d];
    }
    // adjacency
    const int64_t nv = info.col_end[0] - info.col_begin[0];
    cudaMemsetAsync(S.deg, 0, sizeof(int32_t) * (nv + 1), s);
    k_degree<<<gridn(info.col_end[1] - info.col_begin[1], 256), 256, 0, s>>>(info.col_begin[1], info.col_end[1],
                                                                            S.tup[1], dropped, S.deg);
    const int32_t* deg = S.deg;
    int64_t* adj_off = S.adj_off;
    scan([=] __device__(int64_t v) -> int64_t { return v < nv ? deg[v] : 0; },
         [=] __device__(int64_t v, int64_t pre, int64_t) { adj_off[v] = pre; }, nv + 1, S.blk, s);
    cudaMemsetAsync(S.deg, 0, sizeof(int32_t) * (nv + 1), s);
    const bool masks = max_iteration <= kMaskCandidates;
    k_adj_fill<<<gridn(info.col_end[1] - info.col_begin[1], 256), 256, 0, s>>>(
        info.col_begin[1], info.col_end[1], S.tup[1], dropped, S.adj_off, S.deg, S.adj, masks ? S.adj_src : nullptr);
    k_adj_sort<<<gridn(nv, 128), 128, 0, s>>>(nv, S.adj_off, S.adj);
    launches += 6;
    const int64_t ne2 = 2 * int64_t(info.col_end[1] - info.col_begin[1]);  // list entries, at most
    if (masks) {
        k_adj_masks<<<gridn(ne2, 256), 256, 0, s>>>(nv, S.adj_src, S.adj, S.adj_off, max_iteration, S.nmask);
        launches++;
    }
    // hash of the top-dimension tuples
    cudaMemsetAsync(S.table, 0xff, sizeof(int32_t) * (size_t(S.mask) + 1), s);
    const int32_t cb = info.col_begin[top], ce = info.col_end[top];
    k_hash_insert<<<gridn(ce - cb, 256), 256, 0, s>>>(cb, ce, top + 1, S.tup[top], dropped, S.table, S.mask);
    if (masks) {
        k_highclear_masks<<<gridn(ce - cb, 256), 256, 0, s>>>(cb, ce, top, S.tup[top], S.adj, S.adj_off, S.nmask,
                                                             S.table, S.mask, dropped, D.cleared, D.counters);
        return launches + 2;
    }
    const int g = max_iteration <= 4 ? 4 : max_iteration <= 8 ? 8 : max_iteration <= 16 ? 16 : 32;
    const unsigned grid = gridn(int64_t(ce - cb) * g, kHcThreads, 148 * 64);
#define SSPP_HC(G_)                                                                                               \
    k_highclear<G_><<<grid, kHcThreads, 0, s>>>(cb, ce, top, max_iteration, S.tup[top], S.adj, S.adj_off, S.table, S.mask, \
                                         dropped, D.cleared, D.counters)
    if (g == 4) SSPP_HC(4);
    else if (g == 8) SSPP_HC(8);
    else if (g == 16) SSPP_HC(16);
    else SSPP_HC(32);
#undef SSPP_HC
    launches += 2;
    return launches;
}

}  // namespace sspp
