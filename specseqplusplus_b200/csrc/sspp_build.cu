// Filtered flag complexes built on the device, written as boundary matrices.
//
// The reference takes its complexes from external tools (Dionysus / CGAL
// writers, phat-highclear/addons/rips.cpp and alpha_3.cpp) through PHAT files
// (src/main.cu:90-167).  Here the complex is built where it is reduced, so a
// request ships a point cloud or a scalar field (a few MB) instead of its
// boundary matrix (tens of MB for a 64^3 grid).
//
// Both builders produce a flag complex: the Rips complex is the clique complex
// of the graph of pairs at distance <= radius, and the Freudenthal (Kuhn)
// triangulation of a grid is the clique complex of its edge graph (vertices
// joined when their offset is a non-zero 0/1 vector; a clique is a chain in
// the componentwise order, which is a Kuhn simplex).  A simplex's value is the
// largest of its edges' values (Rips: float32 length; lower-star: the larger
// vertex value), vertices have value 0 (Rips) or the field value (lower-star).
//
// Layout.  Vertices 0..V-1.  Edges are the concatenated upper adjacency lists
// (vertex i's neighbours j > i, ascending), so edge ids are in lexicographic
// order.  Triangles (i,j,k) are numbered edge (i,j) by edge, third vertex k
// ascending, found by merging the lists of i (after j) and j; tetrahedra
// (i,j,k,l) triangle by triangle, merging the triangles of edge (i,j) after k
// with the list of k.  Every list comes out in lexicographic order by
// construction, and every facet's id is known from the merge positions (one
// binary search in a short triangle segment for two of a tetrahedron's
// facets).  The global column order (value, dimension, tuple) is one stable
// radix sort of the 32-bit value keys over the concatenation (vertices, edges,
// triangles, tetrahedra), which is already in (dimension, tuple) order.
//
// Floating point is reproduced exactly: distances are summed in coordinate
// order with round-to-nearest and no contraction (__fadd_rn / __fmul_rn,
// __fsqrt_rn), maxima are of bitwise-canonical values (-0 is stored as +0 and
// NaN is rejected), so the matrix equals the host builder's bit for bit.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>

#include "sspp_build.h"
#include "sspp_scan.cuh"

namespace sspp {
namespace {

constexpr int kT = 256;

unsigned grid_for(int64_t n, int64_t cap = 1 << 16) {
    int64_t g = (n + kT - 1) / kT;
    return unsigned(std::max<int64_t>(1, std::min(g, cap)));
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

__device__ __forceinline__ uint32_t fkey(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fval(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
// max with the host's std::max semantics; on canonical values any order gives the same bits
__device__ __forceinline__ float vmax(float a, float b) { return (a < b) ? b : a; }

template <class T>
cudaError_t take(BuildScratch& S, int slot, int64_t count, cudaStream_t s, T** out) {
    const size_t want = std::max<size_t>(sizeof(T) * size_t(std::max<int64_t>(count, 1)), 256);
    if (S.cap[slot] < want) {
        if (S.p[slot]) cudaFreeAsync(S.p[slot], s);
        S.p[slot] = nullptr;
        S.cap[slot] = 0;
        const size_t grown = want + want / 4;
        cudaError_t e = cudaMallocAsync(&S.p[slot], grown, s);
        if (e != cudaSuccess) {
            S.p[slot] = nullptr;
            return e;
        }
        S.cap[slot] = grown;
    }
    *out = static_cast<T*>(S.p[slot]);
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// vertex values: canonical copy (NaN rejected, -0 stored as +0)

__global__ void k_canon(const float* in, float* out, int64_t n, int* flag) {
    GRID_STRIDE(i, n) {
        float v = in[i];
        if (v != v) atomicOr(flag, 1);
        out[i] = (v == 0.0f) ? 0.0f : v;
    }
}

// ---------------------------------------------------------------------------
// Freudenthal grid: upper adjacency

struct Grid {
    int64_t gx, gy, gz;
};

__device__ __forceinline__ int ls_degree(Grid g, int64_t v) {
    const int64_t x = v % g.gx, y = (v / g.gx) % g.gy, z = v / (g.gx * g.gy);
    const int bits = int(x + 1 < g.gx) + int(y + 1 < g.gy) + int(z + 1 < g.gz);
    return (1 << bits) - 1;
}

struct GridDegree {
    Grid g;
    __device__ int64_t operator()(int64_t v) const { return ls_degree(g, v); }
};

__global__ void k_ls_fill(Grid g, const float* val, const int64_t* up_off, int32_t* up_v, float* up_w) {
    const int64_t nv = g.gx * g.gy * g.gz;
    GRID_STRIDE(v, nv) {
        const int64_t x = v % g.gx, y = (v / g.gx) % g.gy, z = v / (g.gx * g.gy);
        int32_t nb[7];
        int m = 0;
        for (int a = 1; a < 8; a++) {
            const int64_t x1 = x + (a & 1), y1 = y + ((a >> 1) & 1), z1 = z + ((a >> 2) & 1);
            if (x1 >= g.gx || y1 >= g.gy || z1 >= g.gz) continue;
            const int32_t u = int32_t((z1 * g.gy + y1) * g.gx + x1);
            int q = m++;
            while (q > 0 && nb[q - 1] > u) {  // ascending (the offsets already grow with the mask)
                nb[q] = nb[q - 1];
                q--;
            }
            nb[q] = u;
        }
        const int64_t o = up_off[v];
        const float fv = val[v];
        for (int q = 0; q < m; q++) {
            up_v[o + q] = nb[q];
            up_w[o + q] = vmax(fv, val[nb[q]]);
        }
    }
}

// ---------------------------------------------------------------------------
// Rips: bounding box, cell sort, neighbour search

__global__ void k_bbox(const float* p, int64_t n, int D, uint32_t* bb, int* flag) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
    bool bad = false;
    GRID_STRIDE(i, n) {
        for (int d = 0; d < D; d++) {
            const float x = p[i * D + d];
            if (!isfinite(x)) bad = true;
            const uint32_t k = fkey(x);
            lo[d] = min(lo[d], k);
            hi[d] = max(hi[d], k);
        }
    }
    for (int d = 0; d < D; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = min(lo[d], __shfl_xor_sync(0xFFFFFFFFu, lo[d], o));
            hi[d] = max(hi[d], __shfl_xor_sync(0xFFFFFFFFu, hi[d], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bb[d], lo[d]);
            atomicMax(&bb[3 + d], hi[d]);
        }
    }
    if (bad) atomicOr(flag, 1);
}

struct CellGrid {
    double lo[3];
    double side;
    int32_t n[3];
};

__device__ __forceinline__ int32_t cell_coord(const CellGrid& c, int d, float x) {
    const double t = floor((double(x) - c.lo[d]) / c.side);
    const int32_t k = int32_t(t);
    return k < 0 ? 0 : (k >= c.n[d] ? c.n[d] - 1 : k);
}

__global__ void k_cells(const float* p, int64_t n, int D, CellGrid c, uint32_t* cell, int32_t* pt) {
    GRID_STRIDE(i, n) {
        uint32_t id = 0;
        for (int d = D - 1; d >= 0; d--) id = id * uint32_t(c.n[d]) + uint32_t(cell_coord(c, d, p[i * D + d]));
        cell[i] = id;
        pt[i] = int32_t(i);
    }
}

__device__ __forceinline__ int64_t lower_bound_u32(const uint32_t* a, int64_t n, uint32_t key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// FILL = false: counts each point's upper neighbours into up_off[i];
// FILL = true: writes them (unsorted) from up_off[i].
template <bool FILL>
__global__ void k_rips_nbrs(const float* p, int64_t n, int D, CellGrid c, const uint32_t* cell, const int32_t* pt,
                            float radius, int64_t* up_off, int32_t* up_v, float* up_w) {
    GRID_STRIDE(i, n) {
        float pi[3] = {0.f, 0.f, 0.f};
        int32_t ci[3] = {0, 0, 0};
        for (int d = 0; d < D; d++) {
            pi[d] = p[i * D + d];
            ci[d] = cell_coord(c, d, pi[d]);
        }
        int lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = d < D ? max(0, ci[d] - 1) : 0;
            hi[d] = d < D ? min(c.n[d] - 1, ci[d] + 1) : 0;
        }
        int64_t cnt = 0;
        const int64_t base = FILL ? up_off[i] : 0;
        for (int z = lo[2]; z <= hi[2]; z++)
            for (int y = lo[1]; y <= hi[1]; y++)
                for (int x = lo[0]; x <= hi[0]; x++) {
                    uint32_t id = uint32_t(x);
                    if (D >= 2) id += uint32_t(c.n[0]) * uint32_t(y);
                    if (D >= 3) id += uint32_t(c.n[0]) * uint32_t(c.n[1]) * uint32_t(z);
                    for (int64_t m = lower_bound_u32(cell, n, id); m < n && cell[m] == id; m++) {
                        const int32_t j = pt[m];
                        if (j <= i) continue;
                        float s = 0.0f;
                        for (int d = 0; d < D; d++) {
                            const float t = __fsub_rn(pi[d], p[int64_t(j) * D + d]);
                            s = __fadd_rn(s, __fmul_rn(t, t));
                        }
                        const float dist = __fsqrt_rn(s);
                        if (dist <= radius) {
                            if (FILL) {
                                up_v[base + cnt] = j;
                                up_w[base + cnt] = dist;
                            }
                            cnt++;
                        }
                    }
                }
        if (!FILL) up_off[i] = cnt;
    }
}

// ---------------------------------------------------------------------------
// cliques

__global__ void k_edge_src(int64_t nv, const int64_t* up_off, int32_t* e_src) {
    GRID_STRIDE(v, nv) {
        for (int64_t e = up_off[v]; e < up_off[v + 1]; e++) e_src[e] = int32_t(v);
    }
}

// triangles (i, j, k), k > j, over edge e = (i, j)
template <bool FILL>
__global__ void k_tri(int64_t E, const int64_t* up_off, const int32_t* up_v, const float* up_w, const int32_t* e_src,
                      int64_t* tri_off, int32_t* tri_k, int4* tri_f, float* tri_w) {
    GRID_STRIDE(e, E) {
        const int32_t i = e_src[e], j = up_v[e];
        int64_t a = e + 1, b = up_off[j];
        const int64_t ae = up_off[i + 1], be = up_off[j + 1];
        int64_t cnt = 0;
        const int64_t base = FILL ? tri_off[e] : 0;
        const float we = FILL ? up_w[e] : 0.0f;
        while (a < ae && b < be) {
            const int32_t va = up_v[a], vb = up_v[b];
            if (va < vb) {
                a++;
            } else if (va > vb) {
                b++;
            } else {
                if (FILL) {
                    const int64_t t = base + cnt;
                    tri_k[t] = va;
                    tri_f[t] = make_int4(int32_t(e), int32_t(a), int32_t(b), 0);
                    tri_w[t] = vmax(vmax(we, up_w[a]), up_w[b]);
                }
                cnt++;
                a++;
                b++;
            }
        }
        if (!FILL) tri_off[e] = cnt;
    }
}

// the triangle of edge e whose third vertex is l (it exists: every clique's faces do)
__device__ __forceinline__ int32_t tri_of(const int64_t* tri_off, const int32_t* tri_k, int32_t e, int32_t l) {
    int64_t lo = tri_off[e], hi = tri_off[e + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (tri_k[mid] < l) lo = mid + 1;
        else hi = mid;
    }
    return int32_t(lo);
}

// tetrahedra (i, j, k, l), l > k, over triangle t = (i, j, k)
template <bool FILL>
__global__ void k_tet(int64_t T, const int64_t* up_off, const int32_t* up_v, const float* up_w, const int64_t* tri_off,
                      const int32_t* tri_k, const int4* tri_f, const float* tri_w, int64_t* tet_off, int4* tet_f,
                      float* tet_w) {
    GRID_STRIDE(t, T) {
        const int4 f = tri_f[t];
        const int32_t k = tri_k[t];
        int64_t a = t + 1, b = up_off[k];
        const int64_t ae = tri_off[f.x + 1], be = up_off[k + 1];
        int64_t cnt = 0;
        const int64_t base = FILL ? tet_off[t] : 0;
        const float wt = FILL ? tri_w[t] : 0.0f;
        while (a < ae && b < be) {
            const int32_t va = tri_k[a], vb = up_v[b];
            if (va < vb) {
                a++;
            } else if (va > vb) {
                b++;
            } else {
                if (FILL) {
                    const int64_t q = base + cnt;
                    tet_f[q] = make_int4(int32_t(t), int32_t(a), tri_of(tri_off, tri_k, f.y, va),
                                         tri_of(tri_off, tri_k, f.z, va));
                    tet_w[q] = vmax(vmax(wt, tri_w[a]), up_w[b]);
                }
                cnt++;
                a++;
                b++;
            }
        }
        if (!FILL) tet_off[t] = cnt;
    }
}

// ---------------------------------------------------------------------------
// global order and the matrix

struct Sizes {
    int64_t V, E, T, Q;
};

__device__ __forceinline__ int dim_of(const Sizes& z, int64_t c) {
    return c < z.V ? 0 : (c < z.V + z.E ? 1 : (c < z.V + z.E + z.T ? 2 : 3));
}

__global__ void k_keys(Sizes z, const float* vval, const float* up_w, const float* tri_w, const float* tet_w,
                       uint32_t* key, int32_t* idx) {
    const int64_t N = z.V + z.E + z.T + z.Q;
    GRID_STRIDE(c, N) {
        float v;
        if (c < z.V) v = vval ? vval[c] : 0.0f;
        else if (c < z.V + z.E) v = up_w[c - z.V];
        else if (c < z.V + z.E + z.T) v = tri_w[c - z.V - z.E];
        else v = tet_w[c - z.V - z.E - z.T];
        key[c] = fkey(v);
        idx[c] = int32_t(c);
    }
}

__global__ void k_place(int64_t N, Sizes z, const uint32_t* key, const int32_t* perm, int32_t* rank, int32_t* dims,
                        float* values) {
    GRID_STRIDE(g, N) {
        const int32_t c = perm[g];
        rank[c] = int32_t(g);
        dims[g] = dim_of(z, c);
        values[g] = fval(key[g]);
    }
}

struct ColLen {
    const int32_t* dims;
    __device__ int64_t operator()(int64_t g) const { return dims[g] == 0 ? 0 : dims[g] + 1; }
};

// Exclusive prefix into off[i]; the total into off[n].
struct OffSink {
    int64_t* off;
    int64_t n;
    __device__ void operator()(int64_t i, int64_t pre, int64_t v) const {
        off[i] = pre;
        if (i == n - 1) off[n] = pre + v;
    }
};

struct ReadArr {
    const int64_t* a;
    __device__ int64_t operator()(int64_t i) const { return a[i]; }
};

__global__ void k_rows(int64_t N, Sizes z, const int32_t* perm, const int32_t* rank, const int32_t* e_src,
                       const int32_t* up_v, const int4* tri_f, const int4* tet_f, const int64_t* col_ptr,
                       int32_t* rows) {
    GRID_STRIDE(g, N) {
        const int64_t c = perm[g];
        int32_t r[4];
        int k;
        if (c < z.V) {
            continue;
        } else if (c < z.V + z.E) {
            const int64_t e = c - z.V;
            r[0] = rank[e_src[e]];
            r[1] = rank[up_v[e]];
            k = 2;
        } else if (c < z.V + z.E + z.T) {
            const int4 f = tri_f[c - z.V - z.E];
            r[0] = rank[z.V + f.x];
            r[1] = rank[z.V + f.y];
            r[2] = rank[z.V + f.z];
            k = 3;
        } else {
            const int4 f = tet_f[c - z.V - z.E - z.T];
            const int64_t o = z.V + z.E;
            r[0] = rank[o + f.x];
            r[1] = rank[o + f.y];
            r[2] = rank[o + f.z];
            r[3] = rank[o + f.w];
            k = 4;
        }
        for (int a = 1; a < k; a++) {
            const int32_t x = r[a];
            int b = a;
            while (b > 0 && r[b - 1] > x) {
                r[b] = r[b - 1];
                b--;
            }
            r[b] = x;
        }
        const int64_t o = col_ptr[g];
        for (int a = 0; a < k; a++) rows[o + a] = r[a];
    }
}

#define BK(call)                                                       \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) {                                       \
            *err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return -2;                                                 \
        }                                                              \
    } while (0)

int fail(std::string* err, const std::string& msg) {
    *err = msg;
    return -1;
}

// Reads up to 8 int64 values from device memory (one synchronisation).
int read_back(BuildScratch& S, std::initializer_list<const int64_t*> src, int64_t* dst, cudaStream_t s,
              std::string* err) {
    int q = 0;
    for (const int64_t* p : src) BK(cudaMemcpyAsync(S.h_misc + q++, p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    BK(cudaStreamSynchronize(s));
    std::memcpy(dst, S.h_misc, sizeof(int64_t) * size_t(q));
    return 0;
}

// Reads the device error flag (one synchronisation); non-zero fails with `what`.
int check_flag(BuildScratch& S, int* flag, cudaStream_t s, std::string* err, const char* what) {
    BK(cudaMemcpyAsync(S.h_misc, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    BK(cudaStreamSynchronize(s));
    int f;
    std::memcpy(&f, S.h_misc, sizeof(int));
    return f ? fail(err, what) : 0;
}

// Exclusive scan of a[0..n) in place, a[n] = total.
int scan_counts(BuildScratch& S, int64_t* a, int64_t n, cudaStream_t s, std::string* err) {
    if (n == 0) {
        BK(cudaMemsetAsync(a, 0, sizeof(int64_t), s));
        return 0;
    }
    int64_t* blk;
    BK(take(S, BuildScratch::BLK, scan_blocks(n) + 2, s, &blk));
    scan(ReadArr{a}, OffSink{a, n}, n, blk, s);
    BK(cudaGetLastError());
    return 0;
}

constexpr int64_t kMaxCols = int64_t(1) << 31;

// Cliques of the graph in S (UP_OFF / UP_V / UP_W over nv vertices), the
// global order and the matrix.
int build_flag(BuildScratch& S, int64_t nv, const float* vval, int maxdim, cudaStream_t s, Built* out,
               std::string* err) {
    const int64_t* up_off = static_cast<const int64_t*>(S.p[BuildScratch::UP_OFF]);
    const int32_t* up_v = static_cast<const int32_t*>(S.p[BuildScratch::UP_V]);
    const float* up_w = static_cast<const float*>(S.p[BuildScratch::UP_W]);
    Sizes z{nv, 0, 0, 0};
    if (maxdim >= 1 && nv > 0) {
        if (read_back(S, {up_off + nv}, &z.E, s, err)) return -2;
    }
    if (z.V + z.E >= kMaxCols) return fail(err, "complex too large (columns >= 2^31)");
    int32_t* e_src = nullptr;
    int32_t* tri_k = nullptr;
    int4* tri_f = nullptr;
    float* tri_w = nullptr;
    int4* tet_f = nullptr;
    float* tet_w = nullptr;
    BK(take(S, BuildScratch::E_SRC, z.E, s, &e_src));
    if (z.E > 0) k_edge_src<<<grid_for(nv), kT, 0, s>>>(nv, up_off, e_src);
    if (maxdim >= 2 && z.E > 0) {
        int64_t* tri_off;
        BK(take(S, BuildScratch::TRI_OFF, z.E + 1, s, &tri_off));
        k_tri<false><<<grid_for(z.E), kT, 0, s>>>(z.E, up_off, up_v, up_w, e_src, tri_off, nullptr, nullptr, nullptr);
        if (scan_counts(S, tri_off, z.E, s, err)) return -2;
        if (read_back(S, {tri_off + z.E}, &z.T, s, err)) return -2;
        if (z.V + z.E + z.T >= kMaxCols) return fail(err, "complex too large (columns >= 2^31)");
        BK(take(S, BuildScratch::TRI_K, z.T, s, &tri_k));
        BK(take(S, BuildScratch::TRI_F, z.T, s, &tri_f));
        BK(take(S, BuildScratch::TRI_W, z.T, s, &tri_w));
        k_tri<true><<<grid_for(z.E), kT, 0, s>>>(z.E, up_off, up_v, up_w, e_src, tri_off, tri_k, tri_f, tri_w);
        if (maxdim >= 3 && z.T > 0) {
            int64_t* tet_off;
            BK(take(S, BuildScratch::TET_OFF, z.T + 1, s, &tet_off));
            k_tet<false><<<grid_for(z.T), kT, 0, s>>>(z.T, up_off, up_v, up_w, tri_off, tri_k, tri_f, tri_w, tet_off,
                                                      nullptr, nullptr);
            if (scan_counts(S, tet_off, z.T, s, err)) return -2;
            if (read_back(S, {tet_off + z.T}, &z.Q, s, err)) return -2;
            if (z.V + z.E + z.T + z.Q >= kMaxCols) return fail(err, "complex too large (columns >= 2^31)");
            BK(take(S, BuildScratch::TET_F, z.Q, s, &tet_f));
            BK(take(S, BuildScratch::TET_W, z.Q, s, &tet_w));
            k_tet<true><<<grid_for(z.T), kT, 0, s>>>(z.T, up_off, up_v, up_w, tri_off, tri_k, tri_f, tri_w, tet_off,
                                                     tet_f, tet_w);
        }
    }
    const int64_t N = z.V + z.E + z.T + z.Q;
    const int64_t nnz = 2 * z.E + 3 * z.T + 4 * z.Q;
    uint32_t *key_a, *key_b;
    int32_t *idx_a, *idx_b, *rank, *dims, *rows;
    int64_t* col_ptr;
    float* values;
    BK(take(S, BuildScratch::KEY_A, N, s, &key_a));
    BK(take(S, BuildScratch::KEY_B, N, s, &key_b));
    BK(take(S, BuildScratch::IDX_A, N, s, &idx_a));
    BK(take(S, BuildScratch::IDX_B, N, s, &idx_b));
    BK(take(S, BuildScratch::RANK, N, s, &rank));
    BK(take(S, BuildScratch::DIMS, N + 1, s, &dims));
    BK(take(S, BuildScratch::COLPTR, N + 1, s, &col_ptr));
    BK(take(S, BuildScratch::ROWS, nnz, s, &rows));
    BK(take(S, BuildScratch::VALUES, N, s, &values));
    if (N > 0) {
        k_keys<<<grid_for(N), kT, 0, s>>>(z, vval, up_w, tri_w, tet_w, key_a, idx_a);
        cub::DoubleBuffer<uint32_t> dk(key_a, key_b);
        cub::DoubleBuffer<int32_t> dv(idx_a, idx_b);
        size_t tmp_bytes = 0;
        BK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dv, int(N), 0, 32, s));
        char* tmp;
        BK(take(S, BuildScratch::TMP, int64_t(tmp_bytes), s, &tmp));
        BK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, dk, dv, int(N), 0, 32, s));
        const uint32_t* key = dk.Current();
        const int32_t* perm = dv.Current();
        k_place<<<grid_for(N), kT, 0, s>>>(N, z, key, perm, rank, dims, values);
        int64_t* blk;
        BK(take(S, BuildScratch::BLK, scan_blocks(N) + 2, s, &blk));
        scan(ColLen{dims}, OffSink{col_ptr, N}, N, blk, s);
        if (nnz > 0)
            k_rows<<<grid_for(N), kT, 0, s>>>(N, z, perm, rank, e_src, up_v, tri_f, tet_f, col_ptr, rows);
    } else {
        BK(cudaMemsetAsync(col_ptr, 0, sizeof(int64_t), s));
    }
    BK(cudaGetLastError());
    out->ncols = N;
    out->nnz = nnz;
    out->dims = dims;
    out->col_ptr = col_ptr;
    out->rows = rows;
    out->values = values;
    return 0;
}

}  // namespace

int build_lowerstar(BuildScratch& S, const float* d_values, int64_t gx, int64_t gy, int64_t gz, int maxdim,
                    cudaStream_t s, Built* out, std::string* err) {
    if (gx < 1 || gy < 1 || gz < 1 || maxdim < 0 || maxdim > 3) return fail(err, "bad grid size or maxdim");
    if (gx > kMaxCols || gy > kMaxCols || gz > kMaxCols || gx * gy > kMaxCols || gx * gy * gz >= kMaxCols / 8)
        return fail(err, "grid too large (vertices >= 2^28)");
    const int64_t nv = gx * gy * gz;
    if (!S.h_misc) BK(cudaMallocHost(&S.h_misc, 8 * sizeof(int64_t)));
    int* flag;
    float* vval;
    int64_t* up_off;
    BK(take(S, BuildScratch::MISC, 8, s, &flag));
    BK(cudaMemsetAsync(flag, 0, sizeof(int), s));
    BK(take(S, BuildScratch::VVAL, nv, s, &vval));
    k_canon<<<grid_for(nv), kT, 0, s>>>(d_values, vval, nv, flag);
    if (check_flag(S, flag, s, err, "NaN vertex value")) return -1;
    BK(take(S, BuildScratch::UP_OFF, nv + 1, s, &up_off));
    int64_t* blk;
    BK(take(S, BuildScratch::BLK, scan_blocks(nv) + 2, s, &blk));
    const Grid g{gx, gy, gz};
    scan(GridDegree{g}, OffSink{up_off, nv}, nv, blk, s);
    int64_t E = 0;
    if (read_back(S, {up_off + nv}, &E, s, err)) return -2;
    int32_t* up_v;
    float* up_w;
    BK(take(S, BuildScratch::UP_V, E, s, &up_v));
    BK(take(S, BuildScratch::UP_W, E, s, &up_w));
    k_ls_fill<<<grid_for(nv), kT, 0, s>>>(g, vval, up_off, up_v, up_w);
    BK(cudaGetLastError());
    return build_flag(S, nv, vval, maxdim, s, out, err);
}

int build_rips(BuildScratch& S, const float* d_points, int64_t npts, int space_dim, float radius, int maxdim,
               cudaStream_t s, Built* out, std::string* err) {
    const int D = space_dim;
    if (npts < 0 || D < 1 || D > 3 || maxdim < 0 || maxdim > 3 || !(radius >= 0.0f) || !std::isfinite(radius))
        return fail(err, "bad point count, space dimension, radius or maxdim");
    if (npts >= kMaxCols / 8) return fail(err, "too many points (>= 2^28)");
    if (!S.h_misc) BK(cudaMallocHost(&S.h_misc, 8 * sizeof(int64_t)));
    int* flag;
    BK(take(S, BuildScratch::MISC, 8, s, &flag));
    int64_t* up_off;
    BK(take(S, BuildScratch::UP_OFF, npts + 1, s, &up_off));
    if (npts == 0 || maxdim == 0) {
        BK(cudaMemsetAsync(up_off, 0, sizeof(int64_t) * size_t(npts + 1), s));
        int32_t* up_v;
        float* up_w;
        BK(take(S, BuildScratch::UP_V, 1, s, &up_v));
        BK(take(S, BuildScratch::UP_W, 1, s, &up_w));
        return build_flag(S, npts, nullptr, maxdim, s, out, err);
    }
    // bounding box (also rejects non-finite coordinates): flag[0] error word,
    // flag[2..4] the smallest keys per axis, flag[5..7] the largest
    uint32_t* bb = reinterpret_cast<uint32_t*>(flag + 2);
    {
        const uint32_t init[8] = {0, 0, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0, 0, 0};
        std::memcpy(S.h_misc, init, sizeof(init));
        BK(cudaMemcpyAsync(flag, S.h_misc, sizeof(init), cudaMemcpyHostToDevice, s));
    }
    k_bbox<<<grid_for(npts, 1024), kT, 0, s>>>(d_points, npts, D, bb, flag);
    if (check_flag(S, flag, s, err, "non-finite point coordinate")) return -1;
    uint32_t hb[6];
    BK(cudaMemcpyAsync(S.h_misc, bb, sizeof(hb), cudaMemcpyDeviceToHost, s));
    BK(cudaStreamSynchronize(s));
    std::memcpy(hb, S.h_misc, sizeof(hb));
    auto kval = [](uint32_t k) {
        uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    };
    // Cells of side > radius (a margin of 2^-10 covers the rounding of the
    // float distance and of the cell coordinate), at most ~1000 per axis.
    CellGrid cg{};
    double ext[3] = {0, 0, 0}, ext_max = 0.0;
    for (int d = 0; d < D; d++) {
        cg.lo[d] = double(kval(hb[d]));
        ext[d] = double(kval(hb[3 + d])) - cg.lo[d];
        ext_max = std::max(ext_max, ext[d]);
    }
    cg.side = std::max({double(radius) * (1.0 + 1.0 / 1024.0), ext_max / 1000.0, 1e-30});
    uint64_t total = 1;
    for (int d = 0; d < 3; d++) {
        cg.n[d] = d < D ? int32_t(std::min(1001.0, std::floor(ext[d] / cg.side) + 1.0)) : 1;
        total *= uint64_t(cg.n[d]);
    }
    int end_bit = 1;
    while (end_bit < 32 && (uint64_t(1) << end_bit) < total) end_bit++;
    uint32_t *cell_a, *cell_b;
    int32_t *pt_a, *pt_b;
    BK(take(S, BuildScratch::CELL_A, npts, s, &cell_a));
    BK(take(S, BuildScratch::CELL_B, npts, s, &cell_b));
    BK(take(S, BuildScratch::PT_A, npts, s, &pt_a));
    BK(take(S, BuildScratch::PT_B, npts, s, &pt_b));
    k_cells<<<grid_for(npts), kT, 0, s>>>(d_points, npts, D, cg, cell_a, pt_a);
    cub::DoubleBuffer<uint32_t> dk(cell_a, cell_b);
    cub::DoubleBuffer<int32_t> dv(pt_a, pt_b);
    size_t tmp_bytes = 0;
    BK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dv, int(npts), 0, end_bit, s));
    char* tmp;
    BK(take(S, BuildScratch::TMP, int64_t(tmp_bytes), s, &tmp));
    BK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, dk, dv, int(npts), 0, end_bit, s));
    const uint32_t* cell = dk.Current();
    const int32_t* pt = dv.Current();
    k_rips_nbrs<false><<<grid_for(npts), kT, 0, s>>>(d_points, npts, D, cg, cell, pt, radius, up_off, nullptr,
                                                      nullptr);
    if (scan_counts(S, up_off, npts, s, err)) return -2;
    int64_t E = 0;
    if (read_back(S, {up_off + npts}, &E, s, err)) return -2;
    if (npts + E >= kMaxCols) return fail(err, "complex too large (columns >= 2^31)");
    int32_t *up_v, *up_v2;
    float *up_w, *up_w2;
    BK(take(S, BuildScratch::UP_V, E, s, &up_v));
    BK(take(S, BuildScratch::UP_W, E, s, &up_w));
    BK(take(S, BuildScratch::UP_V2, E, s, &up_v2));
    BK(take(S, BuildScratch::UP_W2, E, s, &up_w2));
    k_rips_nbrs<true><<<grid_for(npts), kT, 0, s>>>(d_points, npts, D, cg, cell, pt, radius, up_off, up_v2, up_w2);
    if (E > 0) {
        // each vertex's upper neighbours ascending (segmented sort by neighbour id)
        size_t sb = 0;
        BK(cub::DeviceSegmentedSort::StableSortPairs(nullptr, sb, up_v2, up_v, up_w2, up_w, int(E), int(npts), up_off,
                                                     up_off + 1, s));
        BK(take(S, BuildScratch::TMP, int64_t(sb), s, &tmp));
        BK(cub::DeviceSegmentedSort::StableSortPairs(tmp, sb, up_v2, up_v, up_w2, up_w, int(E), int(npts), up_off,
                                                     up_off + 1, s));
    }
    BK(cudaGetLastError());
    return build_flag(S, npts, nullptr, maxdim, s, out, err);
}

cudaError_t build_stage(BuildScratch& S, size_t bytes, cudaStream_t s, void** out) {
    char* p;
    cudaError_t e = take(S, BuildScratch::IN, int64_t(bytes), s, &p);
    *out = p;
    return e;
}

void build_free(BuildScratch& S) {
    for (int q = 0; q < BuildScratch::NUM; q++) {
        if (S.p[q]) cudaFree(S.p[q]);
        S.p[q] = nullptr;
        S.cap[q] = 0;
    }
    if (S.h_misc) cudaFreeHost(S.h_misc);
    S.h_misc = nullptr;
}

}  // namespace sspp
