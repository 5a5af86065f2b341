// ORACLE - test infrastructure only.  C driver around the reference's vendored
// GUDHI edge collapser (include/Flag_complex_edge_collapser.h of the reference,
// compiled from where it lies; nothing is copied).  The edge filtration is the
// edge's position, as in include/specseq.h:210.
#include <cstdint>
#include <tuple>
#include <vector>
#include "Flag_complex_edge_collapser.h"

extern "C" void ref_collapse_edges(int64_t nedges, const int32_t* u, const int32_t* v, uint8_t* out) {
    using E = std::tuple<int32_t, int32_t, float>;
    std::vector<E> g;
    g.reserve(nedges);
    for (int64_t i = 0; i < nedges; i++) g.emplace_back(u[i], v[i], float(g.size()));
    for (int64_t i = 0; i < nedges; i++) out[i] = 0;
    auto rem = Gudhi::collapse::flag_complex_collapse_edges(g);
    // surviving edges keep their original position: the filtration value of
    // the first emission is not needed, only membership (include/specseq.h:420-422)
    std::vector<int64_t> pos;
    for (auto& e : rem) {
        // locate by endpoints: edges are unique
        for (int64_t i = 0; i < nedges; i++)
            if (u[i] == std::get<0>(e) && v[i] == std::get<1>(e)) { out[i] = 1; break; }
    }
}
