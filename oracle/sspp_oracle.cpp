// ORACLE - test infrastructure only.  Not part of the product path.
//
// CPU restatement of the SpecSeq++ reduction semantics, used by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
// Nothing in specseqplusplus_b200/ links or calls this file.
//
// What it restates (reference file:line, relative to the reference project):
//   * PHAT ascii/binary reading          src/main.cu:90-167 (sort + dedup per
//     column; indices kept 0-based here, the reference's +1 shift and dummy
//     column 0 only exist to undo themselves in GetPersistencePairs,
//     include/specseq.h:1182-1193)
//   * dimension-stable reorder           include/specseq.h:439-483
//   * init passes: lowest one, leftmost column per row, apparent pivots,
//     youngest-facet clearing, negative-row compression
//                                         include/kernel.h:444-520
//   * high-dimension guided clearing     include/kernel.h:121-188, 202-292,
//                                         include/specseq.h:215-259, 523-541
//   * Flag-complex edge collapse with edge filtration = edge order and the
//     drop rule for cofaces of dropped edges
//                                         include/Flag_complex_edge_collapser.h:224-482,
//                                         include/specseq.h:209-212, 410-438,
//                                         include/kernel.h:190-198
//   * dualization (anti-transpose, pairs mapped back)
//                                         include/kernel.h:521-580,
//                                         include/specseq.h:303-363, 1188
//   * the reduction itself: twist (clearing) column reduction, dimensions high
//     to low, written from the standard algorithm; PHAT's twist_reduction is
//     the reference's CPU oracle (phat-highclear/src/phat.cpp:149) but PHAT's
//     library headers are not part of the reference tree.
//
// Parity pins: tests/test_oracle.py checks this file against the known-answer
// fixture of the reference (phat-highclear/examples/single_triangle*), against
// an independent dense standard reduction and the rank-based pairing lemma on
// exhaustive small cases, against primal = dual, and (when the reference tree
// is present) the edge collapse against the vendored GUDHI header compiled
// from the reference sources into oracle/_ref/.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

using Col = std::vector<int32_t>;

struct Input {
    int64_t n = 0;
    std::vector<int32_t> dims;
    std::vector<Col> cols;
};

Input make_input(int64_t n, const int32_t* dims, const int64_t* col_ptr, const int32_t* rows) {
    Input in;
    in.n = n;
    in.dims.assign(dims, dims + n);
    in.cols.resize(n);
    for (int64_t j = 0; j < n; j++) in.cols[j].assign(rows + col_ptr[j], rows + col_ptr[j + 1]);
    return in;
}

inline int32_t low_of(const Col& c) { return c.empty() ? -1 : c.back(); }

void sym_diff(const Col& a, const Col& b, Col& out) {
    out.clear();
    out.reserve(a.size() + b.size());
    size_t i = 0, j = 0;
    while (i < a.size() && j < b.size()) {
        if (a[i] < b[j]) out.push_back(a[i++]);
        else if (a[i] > b[j]) out.push_back(b[j++]);
        else { i++; j++; }
    }
    while (i < a.size()) out.push_back(a[i++]);
    while (j < b.size()) out.push_back(b[j++]);
}

// ---------------------------------------------------------------- collapse
// Restatement of the Flag-complex edge collapse (Boissonnat-Pritam, GUDHI's
// Flag_complex_edge_collapser::process_edges).  Edges arrive in filtration
// order; edge e is valid at time t when e < t or e has become critical.  The
// edge uv is dominated at time t when the common neighbourhood C of u and v
// (through valid edges) is non-empty and some w in C is adjacent (through
// valid edges) to every other vertex of C.  A non-dominated arrival becomes
// critical and re-examines, largest index first, the earlier non-critical
// edges that close a triangle with it.
struct Collapser {
    int64_t nv;
    const std::vector<std::pair<int32_t, int32_t>>& edges;
    std::vector<std::vector<std::pair<int32_t, int32_t>>> adj;  // (neighbour, edge id), sorted by neighbour
    std::vector<uint8_t> critical;

    Collapser(int64_t nverts, const std::vector<std::pair<int32_t, int32_t>>& e)
        : nv(nverts), edges(e), adj(nverts), critical(e.size(), 0) {}

    bool valid(int32_t e, int32_t t) const { return e < t || critical[e]; }

    void insert(int32_t e) {
        auto [u, v] = edges[e];
        auto put = [&](int32_t a, int32_t b) {
            auto& r = adj[a];
            auto it = std::lower_bound(r.begin(), r.end(), std::make_pair(b, INT32_MIN));
            r.insert(it, {b, e});
        };
        put(u, v);
        put(v, u);
    }

    // common neighbours of u and v through edges valid at time t
    void common(int32_t u, int32_t v, int32_t t, std::vector<std::pair<int32_t, std::pair<int32_t, int32_t>>>& out) const {
        out.clear();
        const auto& a = adj[u];
        const auto& b = adj[v];
        size_t i = 0, j = 0;
        while (i < a.size() && j < b.size()) {
            if (!valid(a[i].second, t)) { i++; continue; }
            if (!valid(b[j].second, t)) { j++; continue; }
            if (a[i].first < b[j].first) i++;
            else if (a[i].first > b[j].first) j++;
            else { out.push_back({a[i].first, {a[i].second, b[j].second}}); i++; j++; }
        }
    }

    bool adjacent_valid(int32_t w, int32_t x, int32_t t) const {
        const auto& r = adj[w];
        auto it = std::lower_bound(r.begin(), r.end(), std::make_pair(x, INT32_MIN));
        return it != r.end() && it->first == x && valid(it->second, t);
    }

    bool dominated(int32_t e, int32_t t) const {
        std::vector<std::pair<int32_t, std::pair<int32_t, int32_t>>> C;
        common(edges[e].first, edges[e].second, t, C);
        if (C.empty()) return false;
        if (C.size() == 1) return true;
        for (size_t k = 0; k < C.size(); k++) {
            bool ok = true;
            for (size_t m = 0; m < C.size() && ok; m++)
                if (m != k && !adjacent_valid(C[k].first, C[m].first, t)) ok = false;
            if (ok) return true;
        }
        return false;
    }

    void three_cliques(int32_t thresh, int32_t e, std::set<int32_t>& S) const {
        std::vector<std::pair<int32_t, std::pair<int32_t, int32_t>>> C;
        common(edges[e].first, edges[e].second, thresh, C);
        for (auto& c : C) {
            int32_t a = c.second.first, b = c.second.second;
            if (!critical[a] && a < thresh) S.insert(a);
            if (!critical[b] && b < thresh) S.insert(b);
        }
    }

    void run() {
        const int32_t E = int32_t(edges.size());
        for (int32_t t = 0; t < E; t++) {
            insert(t);
            if (t == 0) { critical[0] = 1; continue; }
            if (dominated(t, t)) continue;
            critical[t] = 1;
            std::set<int32_t> S;
            three_cliques(t, t, S);
            while (!S.empty()) {
                auto it = std::prev(S.end());
                int32_t e = *it;
                S.erase(it);
                if (critical[e] || dominated(e, e)) continue;
                critical[e] = 1;
                three_cliques(e, e, S);
            }
        }
    }
};

// Columns removed by the collapse: dropped edges, then every higher simplex
// with a removed facet (include/specseq.h:417-436, include/kernel.h:190-198).
std::vector<uint8_t> collapse_drop(const Input& in) {
    std::vector<uint8_t> drop(in.n, 0);
    std::vector<int32_t> vid(in.n, -1);
    int64_t nv = 0;
    for (int64_t j = 0; j < in.n; j++)
        if (in.dims[j] == 0) vid[j] = int32_t(nv++);
    std::vector<std::pair<int32_t, int32_t>> edges;
    std::vector<int64_t> edge_col;
    for (int64_t j = 0; j < in.n; j++)
        if (in.dims[j] == 1 && in.cols[j].size() == 2) {
            edges.push_back({vid[in.cols[j][0]], vid[in.cols[j][1]]});
            edge_col.push_back(j);
        }
    if (edges.empty()) return drop;
    Collapser cl(nv, edges);
    cl.run();
    for (size_t e = 0; e < edges.size(); e++)
        if (!cl.critical[e]) drop[edge_col[e]] = 1;
    int maxd = 0;
    for (auto d : in.dims) maxd = std::max(maxd, d);
    for (int d = 2; d <= maxd; d++)
        for (int64_t j = 0; j < in.n; j++)
            if (in.dims[j] == d)
                for (int32_t r : in.cols[j])
                    if (drop[r]) { drop[j] = 1; break; }
    return drop;
}

// --------------------------------------------------------------- highclear
// Top-dimension guided clearing.  For a top-dimension simplex s with vertices
// v0 < ... < vD (vertex sets from the first two facets, include/kernel.h:
// 121-188), the candidates w are the neighbours of v0 in ascending order, at
// most max_iteration of them (include/kernel.h:211-213).  A candidate that is
// adjacent to every vertex of s spans t = s + {w}; if every other facet of t
// exists and precedes s, s is the youngest facet of t, so its column is a sum
// of earlier columns and s is positive (include/kernel.h:255-287).
//
// The reference's walk over the neighbour lists compares in the wrong
// direction (include/kernel.h:217), which makes it accept only candidates that
// are the smallest neighbour of every other vertex; this restatement
// intersects the lists as intended.  Both are sound; only the number of
// columns cleared differs, never the persistence pairs.
std::vector<uint8_t> highclear(const Input& in, const std::vector<uint8_t>& drop, int max_iteration) {
    std::vector<uint8_t> cleared(in.n, 0);
    int maxd = 0;
    for (auto d : in.dims) maxd = std::max(maxd, d);
    if (maxd < 1 || max_iteration <= 0) return cleared;
    // vertex tuples
    std::vector<std::vector<int32_t>> verts(in.n);
    for (int d = 0; d <= maxd; d++)
        for (int64_t j = 0; j < in.n; j++) {
            if (in.dims[j] != d) continue;
            if (d == 0) { verts[j] = {int32_t(j)}; continue; }
            const Col& c = in.cols[j];
            if (c.size() < 2) continue;
            std::vector<int32_t> u = verts[c[0]];
            for (int32_t x : verts[c[1]]) u.push_back(x);
            std::sort(u.begin(), u.end());
            u.erase(std::unique(u.begin(), u.end()), u.end());
            verts[j] = u;
        }
    // adjacency (vertex column indices), ascending; edges removed by a collapse are absent
    std::vector<std::vector<int32_t>> nbr(in.n);
    for (int64_t j = 0; j < in.n; j++)
        if (in.dims[j] == 1 && in.cols[j].size() == 2 && !drop[j]) {
            nbr[in.cols[j][0]].push_back(in.cols[j][1]);
            nbr[in.cols[j][1]].push_back(in.cols[j][0]);
        }
    for (auto& l : nbr) std::sort(l.begin(), l.end());
    // top-dimension simplex lookup by vertex tuple
    std::map<std::vector<int32_t>, int64_t> where;
    for (int64_t j = 0; j < in.n; j++)
        if (in.dims[j] == maxd && !drop[j]) where[verts[j]] = j;
    auto has = [&](int32_t a, int32_t b) { return std::binary_search(nbr[a].begin(), nbr[a].end(), b); };
    for (int64_t j = 0; j < in.n; j++) {
        if (in.dims[j] != maxd || drop[j]) continue;
        const auto& s = verts[j];
        if (int(s.size()) != maxd + 1) continue;
        int it = 0;
        for (int32_t w : nbr[s[0]]) {
            if (it++ >= max_iteration) break;
            bool common = true;
            for (size_t i = 1; i < s.size() && common; i++) common = has(s[i], w);
            if (!common) continue;
            bool youngest = true;
            for (size_t i = 0; i < s.size() && youngest; i++) {
                std::vector<int32_t> f;
                for (size_t k = 0; k < s.size(); k++)
                    if (k != i) f.push_back(s[k]);
                f.push_back(w);
                std::sort(f.begin(), f.end());
                auto p = where.find(f);
                if (p == where.end() || p->second > j) youngest = false;
            }
            if (youngest) { cleared[j] = 1; break; }
        }
    }
    return cleared;
}

// ------------------------------------------------------------- init passes
// include/kernel.h:444-520.  leftmost[r] = first column containing row r.  A
// column that is the leftmost column of its lowest row is an apparent pivot
// (no earlier column can ever reach that row).  The lowest row of every
// non-zero column is positive (youngest facet) and its column is cleared.  A
// column that is the leftmost column of any of its rows is negative, and the
// rows of negative simplices are removed from every column.
struct InitState {
    std::vector<int32_t> pivot;       // row -> owning column, -1
    std::vector<uint8_t> cleared;     // zeroed as positive
    std::vector<uint8_t> negative;    // row removed by compression
    std::vector<uint8_t> active;      // needs reduction
};

InitState init_passes(Input& in, const std::vector<uint8_t>& extra_clear) {
    const int64_t n = in.n;
    InitState st;
    st.pivot.assign(n, -1);
    st.cleared.assign(n, 0);
    st.negative.assign(n, 0);
    st.active.assign(n, 0);
    std::vector<int32_t> leftmost(n, INT32_MAX);
    for (int64_t j = 0; j < n; j++)
        for (int32_t r : in.cols[j]) leftmost[r] = std::min(leftmost[r], int32_t(j));
    for (int64_t j = 0; j < n; j++) {
        int32_t l = low_of(in.cols[j]);
        if (l < 0) continue;
        st.cleared[l] = 1;
        if (leftmost[l] == j) st.pivot[l] = int32_t(j);
        for (int32_t r : in.cols[j])
            if (leftmost[r] == j) { st.negative[j] = 1; break; }
    }
    for (int64_t j = 0; j < n; j++)
        if (extra_clear[j]) st.cleared[j] = 1;
    for (int64_t j = 0; j < n; j++) {
        if (st.cleared[j]) { in.cols[j].clear(); continue; }
        Col& c = in.cols[j];
        c.erase(std::remove_if(c.begin(), c.end(), [&](int32_t r) { return st.negative[r] != 0; }), c.end());
    }
    for (int64_t j = 0; j < n; j++) {
        int32_t l = low_of(in.cols[j]);
        st.active[j] = (l >= 0 && st.pivot[l] != int32_t(j)) ? 1 : 0;
    }
    return st;
}

// -------------------------------------------------------------- reduction
struct Stats {
    std::vector<int32_t> adds_per_col;  // additions performed on each column
    int64_t additions = 0;
    int64_t add_bytes = 0;      // sum over additions of 4 * (|a| + |b| + |a xor b|)
    int64_t active_after_init = 0;
    int64_t cleared_init = 0;
    int64_t apparent = 0;
    int64_t highclear = 0;
    int64_t dropped = 0;
};

// Twist reduction of in.cols, dimensions from high to low (or low to high for
// a dual matrix).  Columns already owning a pivot in `pivot` are not touched.
void twist(Input& in, std::vector<int32_t>& pivot, std::vector<uint8_t>& zeroed, bool ascending, Stats& s) {
    int maxd = 0;
    for (auto d : in.dims) maxd = std::max(maxd, d);
    std::vector<std::vector<int64_t>> by_dim(maxd + 1);
    for (int64_t j = 0; j < in.n; j++) by_dim[in.dims[j]].push_back(j);
    Col tmp;
    for (int k = 0; k <= maxd; k++) {
        int d = ascending ? k : maxd - k;
        for (int64_t j : by_dim[d]) {
            if (zeroed[j]) continue;
            Col& c = in.cols[j];
            int32_t l = low_of(c);
            if (l >= 0 && pivot[l] == int32_t(j)) continue;
            while (l >= 0 && pivot[l] >= 0) {
                const Col& p = in.cols[pivot[l]];
                sym_diff(c, p, tmp);
                s.additions++;
                if (!s.adds_per_col.empty()) s.adds_per_col[j]++;
                s.add_bytes += 4 * int64_t(c.size() + p.size() + tmp.size());
                c.swap(tmp);
                l = low_of(c);
            }
            if (l >= 0) {
                pivot[l] = int32_t(j);
                zeroed[l] = 1;           // twist: the lowest row's column is positive
                in.cols[l].clear();
            }
        }
    }
}

Input dual_of(const Input& in) {
    Input out;
    out.n = in.n;
    out.dims.resize(in.n);
    out.cols.assign(in.n, Col());
    for (int64_t j = 0; j < in.n; j++) out.dims[in.n - 1 - j] = in.dims[j];
    for (int64_t j = 0; j < in.n; j++)
        for (int32_t r : in.cols[j]) out.cols[in.n - 1 - r].push_back(int32_t(in.n - 1 - j));
    for (auto& c : out.cols) std::sort(c.begin(), c.end());
    return out;
}

struct Result {
    std::vector<std::pair<int64_t, int64_t>> pairs;
    std::vector<int64_t> essential;
    std::vector<uint8_t> dropped;
    std::vector<uint8_t> highcleared;
    InitState init;
    Stats stats;
};

// model bit 1: high-dimension guided clearing; bit 2: edge collapse.
// preprocess: run the engine's init passes (and highclear) before the twist
// reduction; the pairs are identical either way, the addition trace is not.
Result run(const Input& original, int dualize, int model, int max_iteration, int preprocess) {
    Result R;
    Input in = original;
    const int64_t n = in.n;
    R.stats.adds_per_col.assign(n, 0);
    R.dropped.assign(n, 0);
    if (model & 2) {
        R.dropped = collapse_drop(in);
        for (int64_t j = 0; j < n; j++)
            if (R.dropped[j]) { in.cols[j].clear(); R.stats.dropped++; }
    }
    R.highcleared.assign(n, 0);
    if ((model & 1) && preprocess) {
        R.highcleared = highclear(in, R.dropped, max_iteration);
        for (auto h : R.highcleared) R.stats.highclear += h;
    }
    std::vector<int32_t> pivot(n, -1);
    std::vector<uint8_t> zeroed(n, 0);
    if (preprocess) {
        R.init = init_passes(in, R.highcleared);
        pivot = R.init.pivot;
        for (int64_t j = 0; j < n; j++) {
            zeroed[j] = R.init.cleared[j];
            R.stats.cleared_init += R.init.cleared[j];
            R.stats.active_after_init += R.init.active[j];
            if (R.init.pivot[j] >= 0) R.stats.apparent++;
        }
    }
    if (dualize) {
        Input dual = dual_of(in);
        std::vector<int32_t> dpivot(n, -1);
        std::vector<uint8_t> dzero(n, 0);
        // primal pivots become dual pivots: (low l, col c) -> (low n-1-c, col n-1-l);
        // primal negative columns are dual positive columns (cleared)
        for (int64_t l = 0; l < n; l++)
            if (pivot[l] >= 0) {
                dpivot[n - 1 - pivot[l]] = int32_t(n - 1 - l);
                dzero[n - 1 - pivot[l]] = 1;
            }
        twist(dual, dpivot, dzero, true, R.stats);
        for (int64_t l = 0; l < n; l++)
            if (dpivot[l] >= 0) R.pairs.push_back({n - 1 - dpivot[l], n - 1 - l});
    } else {
        twist(in, pivot, zeroed, false, R.stats);
        for (int64_t l = 0; l < n; l++)
            if (pivot[l] >= 0) R.pairs.push_back({l, pivot[l]});
    }
    std::sort(R.pairs.begin(), R.pairs.end());
    std::vector<uint8_t> paired(n, 0);
    for (auto& p : R.pairs) paired[p.first] = paired[p.second] = 1;
    for (int64_t j = 0; j < n; j++)
        if (!paired[j] && !R.dropped[j]) R.essential.push_back(j);
    return R;
}

// ----------------------------------------------------------------- reader
// src/main.cu:90-167: ascii lines are right-trimmed, blank lines and lines
// starting with '#' are skipped, the first integer is the dimension and the
// rest are face indices; binary is int64 ncols then per column int64 dim,
// int64 count, count int64 indices.  Each column is sorted and de-duplicated.
bool read_phat(const char* path, int binary, Input& in) {
    in = Input();
    if (!binary) {
        std::ifstream f(path);
        if (!f) return false;
        std::string line;
        while (std::getline(f, line)) {
            size_t e = line.find_last_not_of(" \t\n\r\f\v");
            line.erase(e == std::string::npos ? 0 : e + 1);
            if (line.empty() || line[0] == '#') continue;
            std::stringstream ss(line);
            int64_t d;
            ss >> d;
            Col c;
            int64_t x;
            while (ss >> x) c.push_back(int32_t(x));
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            in.dims.push_back(int32_t(d));
            in.cols.push_back(c);
        }
    } else {
        std::ifstream f(path, std::ios::binary);
        if (!f) return false;
        int64_t nc = 0;
        f.read(reinterpret_cast<char*>(&nc), 8);
        if (!f || nc < 0) return false;
        for (int64_t j = 0; j < nc; j++) {
            int64_t d = 0, k = 0;
            f.read(reinterpret_cast<char*>(&d), 8);
            f.read(reinterpret_cast<char*>(&k), 8);
            if (!f || k < 0) return false;
            std::vector<int64_t> v(k);
            f.read(reinterpret_cast<char*>(v.data()), 8 * k);
            if (!f) return false;
            Col c(v.begin(), v.end());
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            in.dims.push_back(int32_t(d));
            in.cols.push_back(c);
        }
    }
    in.n = int64_t(in.cols.size());
    return true;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
struct oracle_result {
    Result r;
};
struct oracle_matrix {
    Input in;
};

extern "C" {

oracle_result* oracle_run(int64_t n, const int32_t* dims, const int64_t* col_ptr, const int32_t* rows, int32_t dualize,
                          int32_t model, int32_t max_iteration, int32_t preprocess) {
    Input in = make_input(n, dims, col_ptr, rows);
    auto* h = new oracle_result;
    h->r = run(in, dualize, model, max_iteration, preprocess);
    return h;
}

int64_t oracle_num_pairs(const oracle_result* h) { return int64_t(h->r.pairs.size()); }
int64_t oracle_num_essential(const oracle_result* h) { return int64_t(h->r.essential.size()); }

void oracle_pairs(const oracle_result* h, int64_t* out) {
    for (size_t i = 0; i < h->r.pairs.size(); i++) {
        out[2 * i] = h->r.pairs[i].first;
        out[2 * i + 1] = h->r.pairs[i].second;
    }
}

void oracle_essential(const oracle_result* h, int64_t* out) {
    std::copy(h->r.essential.begin(), h->r.essential.end(), out);
}

// flags per column: bit0 dropped by collapse, bit1 cleared by highclear,
// bit2 cleared by the init passes, bit3 negative (row compressed),
// bit4 active after init.  apparent[j] = owning column of row j or -1.
void oracle_flags(const oracle_result* h, uint8_t* flags, int32_t* apparent) {
    const Result& r = h->r;
    const int64_t n = int64_t(r.dropped.size());
    for (int64_t j = 0; j < n; j++) {
        uint8_t f = 0;
        if (r.dropped[j]) f |= 1;
        if (r.highcleared[j]) f |= 2;
        if (!r.init.cleared.empty()) {
            if (r.init.cleared[j]) f |= 4;
            if (r.init.negative[j]) f |= 8;
            if (r.init.active[j]) f |= 16;
        }
        flags[j] = f;
        if (apparent) apparent[j] = r.init.pivot.empty() ? -1 : r.init.pivot[j];
    }
}

// additions, add_bytes, active_after_init, cleared_init, apparent, highclear, dropped
void oracle_stats(const oracle_result* h, int64_t* out7) {
    const Stats& s = h->r.stats;
    out7[0] = s.additions;
    out7[1] = s.add_bytes;
    out7[2] = s.active_after_init;
    out7[3] = s.cleared_init;
    out7[4] = s.apparent;
    out7[5] = s.highclear;
    out7[6] = s.dropped;
}

// per-column addition counts of the twist reduction (column index of the
// reduced matrix: input order, or dual order when dualized)
void oracle_adds_per_col(const oracle_result* h, int32_t* out) {
    std::copy(h->r.stats.adds_per_col.begin(), h->r.stats.adds_per_col.end(), out);
}

void oracle_free(oracle_result* h) { delete h; }

// Surviving-edge flags of the collapse for an edge list given in filtration
// order as vertex pairs (u[i], v[i]); out[i] = 1 when edge i survives.
void oracle_collapse_edges(int64_t nverts, int64_t nedges, const int32_t* u, const int32_t* v, uint8_t* out) {
    std::vector<std::pair<int32_t, int32_t>> e(nedges);
    for (int64_t i = 0; i < nedges; i++) e[i] = {u[i], v[i]};
    if (nedges == 0) return;
    Collapser c(nverts, e);
    c.run();
    for (int64_t i = 0; i < nedges; i++) out[i] = c.critical[i];
}

oracle_matrix* oracle_read_phat(const char* path, int32_t binary) {
    auto* h = new oracle_matrix;
    if (!read_phat(path, binary, h->in)) { delete h; return nullptr; }
    return h;
}
int64_t oracle_matrix_ncols(const oracle_matrix* h) { return h->in.n; }
int64_t oracle_matrix_nnz(const oracle_matrix* h) {
    int64_t s = 0;
    for (auto& c : h->in.cols) s += int64_t(c.size());
    return s;
}
void oracle_matrix_copy(const oracle_matrix* h, int32_t* dims, int64_t* col_ptr, int32_t* rows) {
    int64_t p = 0;
    for (int64_t j = 0; j < h->in.n; j++) {
        dims[j] = h->in.dims[j];
        col_ptr[j] = p;
        for (int32_t r : h->in.cols[j]) rows[p++] = r;
    }
    col_ptr[h->in.n] = p;
}
void oracle_matrix_free(oracle_matrix* h) { delete h; }

}  // extern "C"
