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
// Inputs this large explore only once their class has run kExploreMinRuns
// times (a repeated workload, where what is learnt pays back): a poor
// candidate on a one-off large input (a dual reduction of a large lower-star
// grid takes four times as long) costs more than it could teach.  Until then
// they take the lowest estimate: their own class's mean where measured, else
// what similar smaller classes measured.
constexpr int64_t kExploreMaxCols = int64_t(1) << 20;
constexpr int64_t kExploreMinRuns = 2;

struct Entry {
    std::vector<double> mean;   // ms per million columns
    std::vector<int64_t> runs;
    std::vector<int64_t> last;  // run index of the last measurement
    int64_t total = 0;
    double fill = 0;
};

// size class (log2 columns), shape, model, dualize as asked, allow_dual
using Key = std::tuple<int, int, int, int, int>;

std::mutex g_mu;
std::map<Key, Entry>& table() {
    static std::map<Key, Entry> t;
    return t;
}

Key key_of(int64_t ncols, int32_t shape, int32_t model, int32_t dualize, int32_t allow_dual) {
    int lg = 0;
    while ((int64_t(1) << (lg + 1)) <= std::max<int64_t>(ncols, 1)) lg++;
    return Key{lg, shape, model, allow_dual ? 2 : dualize, allow_dual};
}

bool similar(const Key& a, const Key& b) {  // every field but the size
    return std::get<1>(a) == std::get<1>(b) && std::get<2>(a) == std::get<2>(b) && std::get<3>(a) == std::get<3>(b) &&
           std::get<4>(a) == std::get<4>(b);
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

// running mean per candidate over the measured classes similar to k (their
// own means weighted by runs); infinity where none measured it
std::vector<double> prior_of(const Key& k, int n) {
    std::vector<double> sum(size_t(n), 0.0), w(size_t(n), 0.0), out(size_t(n), HUGE_VAL);
    for (const auto& kv : table()) {
        if (kv.first == k || !similar(kv.first, k)) continue;
        for (int c = 0; c < n && c < int(kv.second.mean.size()); c++)
            if (kv.second.runs[size_t(c)] > 0) {
                sum[size_t(c)] += kv.second.mean[size_t(c)];
                w[size_t(c)] += 1.0;
            }
    }
    for (int c = 0; c < n; c++)
        if (w[size_t(c)] > 0) out[size_t(c)] = sum[size_t(c)] / w[size_t(c)];
    return out;
}

}  // namespace

int tune_choose(int64_t ncols, int32_t shape, int32_t model, int32_t dualize, int32_t allow_dual, Knobs* out,
                bool explore_large) {
    std::lock_guard<std::mutex> l(g_mu);
    const Key k = key_of(ncols, shape, model, dualize, allow_dual);
    Entry& e = entry_of(k, allow_dual);
    const int n = int(e.mean.size());
    int pick = -1;
    // untried candidates, best first by what similar classes measured; those
    // over twice as slow there as the best are left out of the first round
    const std::vector<double> prior = prior_of(k, n);
    if (ncols >= kExploreMaxCols && (!explore_large || e.total < kExploreMinRuns)) {
        double bv = HUGE_VAL;
        for (int c = 0; c < n; c++) {
            const double v = e.runs[size_t(c)] > 0 ? e.mean[size_t(c)] : prior[size_t(c)];
            if (v < bv) {
                bv = v;
                pick = c;
            }
        }
        if (pick < 0) pick = 0;  // nothing measured yet: the first candidate (best on the measured workloads)
        *out = kCandidates[pick % kNumBase];
        out->dualize = allow_dual ? (pick >= kNumBase ? 2 : 0) : dualize;
        return pick;
    }
    double best_prior = HUGE_VAL;
    for (double v : prior) best_prior = std::min(best_prior, v);
    for (int c = 0; c < n; c++) {
        if (e.runs[size_t(c)] > 0) continue;
        // measured slow on similar inputs: over twice the best, or a quarter more on large inputs
        const double slack = ncols >= kExploreMaxCols ? 1.25 : 2.0;
        if (std::isfinite(prior[size_t(c)]) && prior[size_t(c)] > slack * best_prior) continue;
        if (pick < 0 || prior[size_t(c)] < prior[size_t(pick)]) pick = c;
    }
    if (pick < 0 && e.total % kRetryEvery == kRetryEvery - 1) {
        pick = 0;  // least recently measured
        for (int c = 1; c < n; c++)
            if (e.last[size_t(c)] < e.last[size_t(pick)]) pick = c;
    }
    if (pick < 0) {
        pick = -1;
        for (int c = 0; c < n; c++)
            if (e.runs[size_t(c)] > 0 && (pick < 0 || e.mean[size_t(c)] < e.mean[size_t(pick)])) pick = c;
        if (pick < 0) pick = 0;
    }
    *out = kCandidates[pick % kNumBase];
    out->dualize = allow_dual ? (pick >= kNumBase ? 2 : 0) : dualize;
    return pick;
}

void tune_record(int64_t ncols, int32_t shape, int32_t model, int32_t dualize, int32_t allow_dual, int cand,
                 double ms, double arena_fill) {
    std::lock_guard<std::mutex> l(g_mu);
    Entry& e = entry_of(key_of(ncols, shape, model, dualize, allow_dual), allow_dual);
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
    // the largest fill seen for this size with these settings, any shape; else any size
    double same = 0, any = 0;
    const Key k = key_of(ncols, 0, model, dualize, allow_dual);
    for (const auto& kv : table()) {
        if (std::get<2>(kv.first) != std::get<2>(k) || std::get<3>(kv.first) != std::get<3>(k) ||
            std::get<4>(kv.first) != std::get<4>(k))
            continue;
        any = std::max(any, kv.second.fill);
        if (std::get<0>(kv.first) == std::get<0>(k)) same = std::max(same, kv.second.fill);
    }
    return same > 0 ? same : (any > 0 ? any : fallback);
}

}  // namespace sspp
