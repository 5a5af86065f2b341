// Synthetic filtered complexes written as PHAT boundary matrices.
//
// These builders produce the inputs the engine is measured and tested on:
//   * Vietoris-Rips complexes of point clouds (seeded uniform in [0,1]^D, or
//     the caller's, D = 1..3), Euclidean float32 distances, truncated at a
//     radius, simplices up to a maximum dimension;
//   * lower-star filtrations of the Freudenthal (Kuhn) triangulation of a
//     grid whose vertex values are seeded Gaussian white noise smoothed by a
//     Gaussian of width sigma voxels (float32), or the caller's field.
// Columns are ordered by (filtration value, dimension, lexicographic vertex
// tuple), which is the order the reference's inputs use (PHAT files written in
// filtration order, src/main.cu:90-167 reads them column by column).  Face
// indices are int32 and each column lists its facets in ascending order.
//
// The builders are host code on the input side of the reduction; they are not
// part of the measured path.  The engine's device builders (sspp_load_rips,
// sspp_load_lowerstar) produce the same matrices bit for bit.  Everything is deterministic given the seed:
// the random stream is SplitMix64, floating point is plain IEEE float/double
// without contraction (built with -ffp-contract=off).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "sspp_gen.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform float in [0,1) with 24 random bits
    float uniform_f() { return float(next() >> 40) * (1.0f / 16777216.0f); }
    // uniform double in (0,1)
    double uniform_d() { return (double(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    // standard normal via Box-Muller (one value per call, the second discarded)
    double normal() {
        double u1 = uniform_d(), u2 = uniform_d();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// Monotone map float -> uint32 so that unsigned comparison equals float order.
inline uint32_t float_key(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

constexpr int VBITS = 21;  // vertex index width in packed tuples (n < 2^21)

struct Simplex {
    uint32_t vkey;      // float_key(value)
    uint32_t dim;
    uint64_t hi;        // packed vertex tuple, first three vertices (big-endian by position)
    uint32_t lo;        // fourth vertex (tetrahedra), else 0
    uint32_t pad;
    bool operator<(const Simplex& o) const {
        if (vkey != o.vkey) return vkey < o.vkey;
        if (dim != o.dim) return dim < o.dim;
        if (hi != o.hi) return hi < o.hi;
        return lo < o.lo;
    }
};

inline uint64_t pack3(uint32_t a, uint32_t b, uint32_t c) {
    return (uint64_t(a) << (2 * VBITS)) | (uint64_t(b) << VBITS) | uint64_t(c);
}

// A simplex's vertices in ascending order, from its packed form.
inline int unpack(const Simplex& s, uint32_t* v) {
    const uint64_t m = (1ull << VBITS) - 1;
    int k = int(s.dim) + 1;
    if (k <= 3) {
        // stored right-aligned: the k vertices occupy the low k slots
        for (int i = 0; i < k; i++) v[i] = uint32_t((s.hi >> (VBITS * (k - 1 - i))) & m);
    } else {
        v[0] = uint32_t((s.hi >> (2 * VBITS)) & m);
        v[1] = uint32_t((s.hi >> VBITS) & m);
        v[2] = uint32_t(s.hi & m);
        v[3] = s.lo;
    }
    return k;
}

inline Simplex make_simplex(float value, int dim, const uint32_t* v) {
    Simplex s;
    s.vkey = float_key(value);
    s.dim = uint32_t(dim);
    s.pad = 0;
    s.lo = 0;
    switch (dim) {
        case 0: s.hi = v[0]; break;
        case 1: s.hi = (uint64_t(v[0]) << VBITS) | v[1]; break;
        case 2: s.hi = pack3(v[0], v[1], v[2]); break;
        default: s.hi = pack3(v[0], v[1], v[2]); s.lo = v[3]; break;
    }
    return s;
}

inline uint64_t tuple_key(const uint32_t* v, int k) {
    uint64_t key = 0;
    for (int i = 0; i < k; i++) key = (key << VBITS) | v[i];
    return key;
}

struct Matrix {
    std::vector<int32_t> dims;
    std::vector<int64_t> col_ptr;
    std::vector<int32_t> rows;
    std::vector<float> values;
};

// Sorts the simplices into filtration order and writes the boundary matrix.
// Facets (dimension <= 2, at most three vertices) are found by binary search
// in a per-dimension table of (packed tuple, column index).
void build_matrix(std::vector<Simplex>& sx, Matrix& out) {
    std::sort(sx.begin(), sx.end());
    const int64_t n = int64_t(sx.size());
    std::vector<std::vector<std::pair<uint64_t, int32_t>>> table(3);
    for (int64_t i = 0; i < n; i++) {
        if (sx[i].dim <= 2) table[sx[i].dim].push_back({sx[i].hi, int32_t(i)});
    }
    for (auto& t : table) std::sort(t.begin(), t.end());
    out.dims.resize(n);
    out.values.resize(n);
    out.col_ptr.assign(n + 1, 0);
    int64_t nnz = 0;
    for (int64_t i = 0; i < n; i++) nnz += (sx[i].dim == 0) ? 0 : int64_t(sx[i].dim) + 1;
    out.rows.resize(nnz);
    int64_t p = 0;
    for (int64_t i = 0; i < n; i++) {
        const Simplex& s = sx[i];
        out.dims[i] = int32_t(s.dim);
        uint32_t key = s.vkey;
        uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
        float f;
        std::memcpy(&f, &u, 4);
        out.values[i] = f;
        out.col_ptr[i] = p;
        if (s.dim > 0) {
            uint32_t v[4], fv[4];
            int k = unpack(s, v);
            int32_t faces[4];
            for (int drop = 0; drop < k; drop++) {
                int m = 0;
                for (int j = 0; j < k; j++)
                    if (j != drop) fv[m++] = v[j];
                uint64_t fk = tuple_key(fv, k - 1);
                auto& t = table[k - 2];
                auto it = std::lower_bound(t.begin(), t.end(), std::make_pair(fk, int32_t(-1)));
                faces[drop] = it->second;  // every facet of a generated simplex exists
            }
            std::sort(faces, faces + k);
            for (int j = 0; j < k; j++) out.rows[p++] = faces[j];
        }
    }
    out.col_ptr[n] = p;
}

struct Nbr {
    uint32_t v;
    float d;
};

std::vector<float> gen_points(int64_t npts, int D, uint64_t seed) {
    SplitMix64 rng(seed);
    std::vector<float> P(static_cast<size_t>(npts) * D);
    for (auto& x : P) x = rng.uniform_f();
    return P;
}

// Rips complex of P (npts x D, D in 1..3).  Candidate pairs come from a grid
// of cells of side > radius over the points' bounding box (cell coordinates in
// double; at most ~1000 cells per axis), so every pair at float distance <=
// radius lies in the same or adjacent cells whatever the coordinates' range.
void gen_rips(const float* P, int64_t npts, int D, float radius, int maxdim, Matrix& out) {
    double lo[3] = {0, 0, 0}, ext[3] = {0, 0, 0};
    for (int d = 0; d < D; d++) {
        float mn = P[d], mx = P[d];
        for (int64_t i = 1; i < npts; i++) {
            mn = std::min(mn, P[i * D + d]);
            mx = std::max(mx, P[i * D + d]);
        }
        lo[d] = double(mn);
        ext[d] = double(mx) - lo[d];
    }
    const double ext_max = std::max({ext[0], ext[1], ext[2]});
    const double side = std::max({double(radius) * (1.0 + 1.0 / 1024.0), ext_max / 1000.0, 1e-30});
    int32_t ncell[3] = {1, 1, 1};
    for (int d = 0; d < D; d++) ncell[d] = int32_t(std::min(1001.0, std::floor(ext[d] / side) + 1.0));
    auto coord = [&](int d, float x) {
        int32_t k = int32_t(std::floor((double(x) - lo[d]) / side));
        return k < 0 ? 0 : (k >= ncell[d] ? ncell[d] - 1 : k);
    };
    auto cell_id = [&](int32_t x, int32_t y, int32_t z) {
        return (uint64_t(z) * uint64_t(ncell[1]) + uint64_t(y)) * uint64_t(ncell[0]) + uint64_t(x);
    };
    std::vector<std::pair<uint64_t, uint32_t>> members(static_cast<size_t>(npts));
    for (int64_t i = 0; i < npts; i++) {
        int32_t c[3] = {0, 0, 0};
        for (int d = 0; d < D; d++) c[d] = coord(d, P[i * D + d]);
        members[size_t(i)] = {cell_id(c[0], c[1], c[2]), uint32_t(i)};
    }
    std::sort(members.begin(), members.end());
    // upper adjacency: neighbours with larger index, ascending
    std::vector<std::vector<Nbr>> up(static_cast<size_t>(npts));
    for (int64_t i = 0; i < npts; i++) {
        int32_t c[3] = {0, 0, 0};
        for (int d = 0; d < D; d++) c[d] = coord(d, P[i * D + d]);
        int32_t lo_c[3], hi_c[3];
        for (int d = 0; d < 3; d++) {
            lo_c[d] = d < D ? std::max(0, c[d] - 1) : 0;
            hi_c[d] = d < D ? std::min(ncell[d] - 1, c[d] + 1) : 0;
        }
        for (int32_t z = lo_c[2]; z <= hi_c[2]; z++)
            for (int32_t y = lo_c[1]; y <= hi_c[1]; y++)
                for (int32_t x = lo_c[0]; x <= hi_c[0]; x++) {
                    const uint64_t id = cell_id(x, y, z);
                    auto it = std::lower_bound(members.begin(), members.end(), std::make_pair(id, uint32_t(0)));
                    for (; it != members.end() && it->first == id; ++it) {
                        uint32_t j = it->second;
                        if (j <= uint32_t(i)) continue;
                        float s = 0.0f;
                        for (int d = 0; d < D; d++) {
                            float t = P[i * D + d] - P[size_t(j) * D + d];
                            s = s + t * t;
                        }
                        float dist = std::sqrt(s);
                        if (dist <= radius) up[size_t(i)].push_back({j, dist});
                    }
                }
        std::sort(up[size_t(i)].begin(), up[size_t(i)].end(), [](const Nbr& a, const Nbr& b) { return a.v < b.v; });
    }
    std::vector<Simplex> sx;
    sx.reserve(size_t(npts) * 8);
    uint32_t v[4];
    for (int64_t i = 0; i < npts; i++) {
        v[0] = uint32_t(i);
        sx.push_back(make_simplex(0.0f, 0, v));
    }
    auto common = [](const std::vector<Nbr>& a, const std::vector<Nbr>& b, uint32_t above,
                     std::vector<std::pair<uint32_t, float>>& res) {
        // vertices w > above in both lists; res holds (w, max of the two distances)
        res.clear();
        size_t ia = 0, ib = 0;
        while (ia < a.size() && a[ia].v <= above) ia++;
        while (ib < b.size() && b[ib].v <= above) ib++;
        while (ia < a.size() && ib < b.size()) {
            if (a[ia].v < b[ib].v) ia++;
            else if (a[ia].v > b[ib].v) ib++;
            else { res.push_back({a[ia].v, std::max(a[ia].d, b[ib].d)}); ia++; ib++; }
        }
    };
    std::vector<std::pair<uint32_t, float>> c2, c3;
    for (int64_t i = 0; i < npts; i++) {
        for (const Nbr& e : up[size_t(i)]) {
            v[0] = uint32_t(i); v[1] = e.v;
            if (maxdim >= 1) sx.push_back(make_simplex(e.d, 1, v));
            if (maxdim < 2) continue;
            common(up[i], up[e.v], e.v, c2);
            for (auto& w : c2) {
                float f2 = std::max(e.d, w.second);
                v[2] = w.first;
                sx.push_back(make_simplex(f2, 2, v));
                if (maxdim < 3) continue;
                // tetrahedra (i, e.v, w, x) with x > w adjacent to all three
                common(up[i], up[e.v], w.first, c3);
                const std::vector<Nbr>& uw = up[w.first];
                size_t iw = 0;
                for (auto& x : c3) {
                    while (iw < uw.size() && uw[iw].v < x.first) iw++;
                    if (iw < uw.size() && uw[iw].v == x.first) {
                        v[3] = x.first;
                        sx.push_back(make_simplex(std::max(f2, std::max(x.second, uw[iw].d)), 3, v));
                    }
                }
            }
        }
    }
    build_matrix(sx, out);
}

// Separable Gaussian smoothing with scipy.ndimage conventions: truncate at
// 4 sigma (radius = int(4 sigma + 0.5)), normalised weights, 'reflect' mode
// (d c b a | a b c d | d c b a).
void smooth_axis(std::vector<double>& f, int G, int axis, const std::vector<double>& w, int R) {
    std::vector<double> line(G), outl(G);
    int64_t stride = (axis == 0) ? 1 : (axis == 1 ? G : int64_t(G) * G);
    for (int a = 0; a < G; a++)
        for (int b = 0; b < G; b++) {
            int64_t base;
            if (axis == 0) base = (int64_t(b) * G + a) * G;
            else if (axis == 1) base = int64_t(b) * G * G + a;
            else base = int64_t(b) * G + a;
            for (int t = 0; t < G; t++) line[t] = f[base + t * stride];
            for (int t = 0; t < G; t++) {
                double s = 0.0;
                for (int k = -R; k <= R; k++) {
                    int q = t + k;
                    // reflect about the half-sample boundary, repeated as needed
                    int period = 2 * G;
                    q = ((q % period) + period) % period;
                    if (q >= G) q = period - 1 - q;
                    s += w[k + R] * line[q];
                }
                outl[t] = s;
            }
            for (int t = 0; t < G; t++) f[base + t * stride] = outl[t];
        }
}

// Seeded N(0,1) white noise on a G^3 grid (x fastest) smoothed by a Gaussian
// of width sigma voxels, rounded to float32.
std::vector<float> gen_field(int G, float sigma, uint64_t seed) {
    const int64_t NV = int64_t(G) * G * G;
    SplitMix64 rng(seed);
    std::vector<double> f(NV);
    for (auto& x : f) x = rng.normal();
    if (sigma > 0) {
        int R = int(4.0 * sigma + 0.5);
        std::vector<double> w(2 * R + 1);
        double tot = 0;
        for (int k = -R; k <= R; k++) { w[k + R] = std::exp(-0.5 * double(k) * k / (double(sigma) * sigma)); tot += w[k + R]; }
        for (auto& x : w) x /= tot;
        for (int axis = 0; axis < 3; axis++) smooth_axis(f, G, axis, w, R);
    }
    std::vector<float> val(NV);
    for (int64_t i = 0; i < NV; i++) val[i] = float(f[i]);
    return val;
}

// Lower-star filtration of the Freudenthal triangulation of a gx x gy x gz
// grid with vertex values `values` (x fastest; -0 read as +0), simplices up
// to maxdim.
void gen_lowerstar(const float* values, int gx, int gy, int gz, int maxdim, Matrix& out) {
    const int64_t NV = int64_t(gx) * gy * gz;
    std::vector<float> val(values, values + NV);
    for (auto& x : val)
        if (x == 0.0f) x = 0.0f;
    auto idx = [gx, gy](int x, int y, int z) { return uint32_t((int64_t(z) * gy + y) * gx + x); };
    // increments are non-empty subsets of {x,y,z} encoded as bit masks 1..7
    auto step = [&](int mask, int& x, int& y, int& z) -> bool {
        if (mask & 1) x++;
        if (mask & 2) y++;
        if (mask & 4) z++;
        return x < gx && y < gy && z < gz;
    };
    std::vector<Simplex> sx;
    sx.reserve(size_t(NV) * (maxdim >= 3 ? 26 : 8));
    uint32_t v[4];
    for (int z = 0; z < gz; z++)
        for (int y = 0; y < gy; y++)
            for (int x = 0; x < gx; x++) {
                uint32_t v0 = idx(x, y, z);
                v[0] = v0;
                sx.push_back(make_simplex(val[v0], 0, v));
                if (maxdim < 1) continue;
                for (int a = 1; a < 8; a++) {
                    int x1 = x, y1 = y, z1 = z;
                    if (!step(a, x1, y1, z1)) continue;
                    uint32_t v1 = idx(x1, y1, z1);
                    v[1] = v1;
                    float f1 = std::max(val[v0], val[v1]);
                    sx.push_back(make_simplex(f1, 1, v));
                    if (maxdim < 2) continue;
                    for (int b = 1; b < 8; b++) {
                        if (b & a) continue;
                        int x2 = x1, y2 = y1, z2 = z1;
                        if (!step(b, x2, y2, z2)) continue;
                        uint32_t v2 = idx(x2, y2, z2);
                        v[2] = v2;
                        float f2 = std::max(f1, val[v2]);
                        sx.push_back(make_simplex(f2, 2, v));
                        if (maxdim < 3) continue;
                        int c = 7 & ~(a | b);
                        if ((a | b) == 7 || c == 0) continue;
                        int x3 = x2, y3 = y2, z3 = z2;
                        if (!step(c, x3, y3, z3)) continue;
                        // tetrahedra need all three singleton increments
                        if (__builtin_popcount(a) != 1 || __builtin_popcount(b) != 1) continue;
                        uint32_t v3 = idx(x3, y3, z3);
                        v[3] = v3;
                        sx.push_back(make_simplex(std::max(f2, val[v3]), 3, v));
                    }
                }
            }
    build_matrix(sx, out);
}

}  // namespace

struct sspp_gen_matrix {
    Matrix m;
};

extern "C" {

sspp_gen_matrix* sspp_gen_rips(int64_t npts, int32_t space_dim, uint64_t seed, float radius, int32_t maxdim) {
    if (npts <= 0 || npts >= (int64_t(1) << VBITS) || space_dim < 1 || space_dim > 3) return nullptr;
    std::vector<float> P = gen_points(npts, space_dim, seed);
    return sspp_gen_rips_points(npts, space_dim, P.data(), radius, maxdim);
}

sspp_gen_matrix* sspp_gen_rips_points(int64_t npts, int32_t space_dim, const float* points, float radius,
                                      int32_t maxdim) {
    if (npts <= 0 || npts >= (int64_t(1) << VBITS) || space_dim < 1 || space_dim > 3 || maxdim < 0 || maxdim > 3 ||
        !(radius >= 0.0f) || !std::isfinite(radius) || !points)
        return nullptr;
    for (int64_t i = 0; i < npts * space_dim; i++)
        if (!std::isfinite(points[i])) return nullptr;
    auto* h = new (std::nothrow) sspp_gen_matrix;
    if (!h) return nullptr;
    gen_rips(points, npts, space_dim, radius, maxdim, h->m);
    return h;
}

int32_t sspp_gen_points(int64_t npts, int32_t space_dim, uint64_t seed, float* out) {
    if (npts < 0 || space_dim < 1 || !out) return -1;
    std::vector<float> P = gen_points(npts, space_dim, seed);
    std::memcpy(out, P.data(), P.size() * sizeof(float));
    return 0;
}

sspp_gen_matrix* sspp_gen_lowerstar(int32_t grid, float sigma, uint64_t seed) {
    if (grid < 2 || int64_t(grid) * grid * grid >= (int64_t(1) << VBITS) || sigma < 0.0f) return nullptr;
    std::vector<float> val = gen_field(grid, sigma, seed);
    return sspp_gen_lowerstar_field(grid, grid, grid, val.data(), 3);
}

sspp_gen_matrix* sspp_gen_lowerstar_field(int32_t gx, int32_t gy, int32_t gz, const float* values, int32_t maxdim) {
    if (gx < 1 || gy < 1 || gz < 1 || int64_t(gx) * gy * gz >= (int64_t(1) << VBITS) || maxdim < 0 || maxdim > 3 ||
        !values)
        return nullptr;
    for (int64_t i = 0; i < int64_t(gx) * gy * gz; i++)
        if (values[i] != values[i]) return nullptr;
    auto* h = new (std::nothrow) sspp_gen_matrix;
    if (!h) return nullptr;
    gen_lowerstar(values, gx, gy, gz, maxdim, h->m);
    return h;
}

int32_t sspp_gen_field(int32_t grid, float sigma, uint64_t seed, float* out) {
    if (grid < 1 || sigma < 0.0f || !out) return -1;
    std::vector<float> val = gen_field(grid, sigma, seed);
    std::memcpy(out, val.data(), val.size() * sizeof(float));
    return 0;
}

int64_t sspp_gen_ncols(const sspp_gen_matrix* h) { return h ? int64_t(h->m.dims.size()) : -1; }
int64_t sspp_gen_nnz(const sspp_gen_matrix* h) { return h ? int64_t(h->m.rows.size()) : -1; }

int32_t sspp_gen_copy(const sspp_gen_matrix* h, int32_t* dims, int64_t* col_ptr, int32_t* rows, float* values) {
    if (!h) return -1;
    const Matrix& m = h->m;
    if (dims) std::memcpy(dims, m.dims.data(), m.dims.size() * sizeof(int32_t));
    if (col_ptr) std::memcpy(col_ptr, m.col_ptr.data(), m.col_ptr.size() * sizeof(int64_t));
    if (rows) std::memcpy(rows, m.rows.data(), m.rows.size() * sizeof(int32_t));
    if (values) std::memcpy(values, m.values.data(), m.values.size() * sizeof(float));
    return 0;
}

void sspp_gen_free(sspp_gen_matrix* h) { delete h; }

}  // extern "C"
