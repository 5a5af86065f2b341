// Autotuner of the reduction's launch parameters (sspp_params.autotune).
//
// The reference takes ss_block_size, block_size_growth_rate, queue_size and
// the level capacities from its command line (src/main.cu:281-294), set by
// hand per dataset.  Here a process-wide history, keyed by size class (log2 of
// the column count), shape (top dimension and the share of columns in it),
// model, dualization and whether the tuner may choose dualization itself,
// records the measured time of each candidate setting.  A new class first
// tries the candidates in the order of their means over similar classes
// (same key but size), leaving out those over twice as slow there as the best,
// then runs the fastest (by running mean of ms per column), re-trying the least
// recently measured one every 32nd run so that the choice follows drift.
// Inputs of 2^20 columns or more explore only once their class has run twice
// (a repeated workload), and skip candidates a quarter slower than the best on
// similar inputs; before that they take the lowest estimate (their class's own
// mean, else the similar classes'), or the first candidate when nothing is
// known.  Every candidate gives the same pairs; only the time
// differs.  The history also keeps the largest arena fill seen per class
// (arena ints used / base ints), which admission control turns into a
// device-memory estimate.
#pragma once
#include <stdint.h>

namespace sspp {

struct Knobs {
    int32_t ss_block_size;
    float growth;
    int32_t queue_size;
    int32_t level1;
    int32_t level2;
    int32_t heavy_threads;
    int32_t dualize;
};

// allow_dual: the tuner may also choose dualization mode 2 (autotune = 2);
// it never picks the full dual (mode 1), whose vertex columns can carry very
// long addition chains on grid-like complexes
// shape: a coarse description of the complex (top dimension and the share of
// its columns there), so that, e.g., grids and Rips complexes of one size
// class are tuned apart
// explore_large = false: inputs of 2^20 columns or more never explore (a
// context that shares the GPU with others, e.g. a server worker: a slow trial
// there delays every request behind it)
int tune_choose(int64_t ncols, int32_t shape, int32_t model, int32_t dualize, int32_t allow_dual, Knobs* out,
                bool explore_large = true);
void tune_record(int64_t ncols, int32_t shape, int32_t model, int32_t dualize, int32_t allow_dual, int cand,
                 double ms, double arena_fill);
// largest arena fill (used / base) recorded for this class (or, before any
// run of it, for any size with the same settings), or `fallback`
double tune_fill(int64_t ncols, int32_t model, int32_t dualize, int32_t allow_dual, double fallback);

}  // namespace sspp
