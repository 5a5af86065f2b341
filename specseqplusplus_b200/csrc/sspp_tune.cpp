// Autotuner history (see sspp_tune.h).
#include "sspp_tune.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace sspp {

namespace {

// Candidate launch settings, best first on the measured workloads (lower-
// star grids and Rips complexes: one spectral-sequence block over the whole
// dimension and 32-int warp columns were fastest or within a few percent).
// queue_size only caps the light tier's grid, so it is set never to bind.
const Knobs kCandidates[] = {
    {1 << 30, 1.0f, 1 << 20, 32, 8192, 256, 0},
    {102400, 1.05f, 1 << 20, 32, 8192, 256, 0},
    {1 << 30, 1.0f, 1 << 20, 64, 8192, 256, 0},
    {1 << 30, 1.0f, 1 << 20, 32, 4096, 128, 0},
};
constexpr int kNumBase = int(sizeof(kCandidates) / sizeof(kCandidates[0]));
constexpr int kRetryEvery = 32;

struct Entry {
    std::vector<double> mean;   // ms per million columns
    std::vector<int64_t> runs;
    std::vector<int64_t> last;  // run index of the last measurement
    int64_t total = 0;
    double fill = 0;
};

using Key = std::tuple<int, int, int, int>;

std::mutex g_mu;
std::map<Key, Entry>& table() {
    static std::map<Key, Entry> t;
    return t;
}

Key key_of(int64_t ncols, int32_t model, int32_t dualize, int32_t allow_dual) {
    int lg = 0;
    while ((int64_t(1) << (lg + 1)) <= std::max<int64_t>(ncols, 1)) lg++;
    return Key{lg, model, allow_dual ? 2 : dualize, allow_dual};
}

int num_candidates(int32_t allow_dual) { return allow_dual ? 2 * kNumBase : kNumBase; }

Entry& entry_of(const Key& k, int32_t allow_dual) {
    Entry& e = table()[k];
    if (e.mean.empty()) {
        const int n = num_candidates(allow_dual);
        e.mean.assign(size_t(n), 0.0);
        e.runs.assign(size_t(n), 0);
        e.last.assign(size_t(n), -1);
    }
    return e;
}

}  // namespace

int tune_choose(int64_t ncols, int32_t model, int32_t dualize, int32_t allow_dual, Knobs* out) {
    std::lock_guard<std::mutex> l(g_mu);
    Entry& e = entry_of(key_of(ncols, model, dualize, allow_dual), allow_dual);
    const int n = int(e.mean.size());
    int pick = -1;
    for (int c = 0; c < n && pick < 0; c++)
        if (e.runs[size_t(c)] == 0) pick = c;
    if (pick < 0 && e.total % kRetryEvery == kRetryEvery - 1) {
        pick = 0;  // least recently measured
        for (int c = 1; c < n; c++)
            if (e.last[size_t(c)] < e.last[size_t(pick)]) pick = c;
    }
    if (pick < 0) {
        pick = 0;
        for (int c = 1; c < n; c++)
            if (e.mean[size_t(c)] < e.mean[size_t(pick)]) pick = c;
    }
    *out = kCandidates[pick % kNumBase];
    out->dualize = allow_dual ? (pick >= kNumBase ? 2 : 0) : dualize;
    return pick;
}

void tune_record(int64_t ncols, int32_t model, int32_t dualize, int32_t allow_dual, int cand, double ms,
                 double arena_fill) {
    std::lock_guard<std::mutex> l(g_mu);
    Entry& e = entry_of(key_of(ncols, model, dualize, allow_dual), allow_dual);
    if (cand < 0 || cand >= int(e.mean.size()) || !(ms >= 0)) return;
    const double v = ms * 1e6 / double(std::max<int64_t>(ncols, 1));
    const size_t c = size_t(cand);
    e.mean[c] = e.runs[c] == 0 ? v : 0.7 * e.mean[c] + 0.3 * v;
    e.runs[c]++;
    e.last[c] = e.total++;
    if (std::isfinite(arena_fill)) e.fill = std::max(e.fill, arena_fill);
}

double tune_fill(int64_t ncols, int32_t model, int32_t dualize, int32_t allow_dual, double fallback) {
    std::lock_guard<std::mutex> l(g_mu);
    const Key k = key_of(ncols, model, dualize, allow_dual);
    auto it = table().find(k);
    if (it != table().end() && it->second.fill > 0) return it->second.fill;
    // no run of this size class yet: the largest fill of any size with the same settings
    double f = 0;
    for (const auto& kv : table())
        if (std::get<1>(kv.first) == std::get<1>(k) && std::get<2>(kv.first) == std::get<2>(k) &&
            std::get<3>(kv.first) == std::get<3>(k))
            f = std::max(f, kv.second.fill);
    return f > 0 ? f : fallback;
}

}  // namespace sspp
