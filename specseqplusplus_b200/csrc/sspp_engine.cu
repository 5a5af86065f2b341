// Engine context, device memory, orchestration and the C ABI (include/sspp.h).
//
// Reference counterpart: class SpecSeqPlusPlus (include/specseq.h:63-1194):
// constructor + MemAlloc1-4 (device arrays), GPU_Init (init passes, guided
// clearing, collapse, dualization, ColumnShrink), GPU_Compute (spectral-
// sequence loop) and GetPersistencePairs.  Differences by design: all state is
// plain device memory (no managed memory), the host synchronises once after
// the init passes and once after the reduction (the reference synchronises
// after every launch and reads queue counts back every iteration), and no
// column is ever reduced on the host.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "sspp_build.h"
#include "sspp_collapse.h"
#include "sspp_highclear.h"
#include "sspp_internal.h"
#include "sspp_io.h"
#include "sspp_launch.h"
#include "sspp_tune.h"
#include "sspp_xfer.h"

using namespace sspp;

// CTA-tier launches of successive spectral-sequence steps run on separate side
// streams.  The driver maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware
// work queues (8 by default), and launches on streams that share a queue wait
// for each other: a short launch queued behind a long chain of another step.
// When the library is loaded, ask for the maximum (32) unless the variable is
// set; it applies to a CUDA context created afterwards (for a program linked
// against the library, every context).
__attribute__((constructor)) static void sspp_request_hw_queues() {
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
}

namespace {
enum Phase { PH_INIT = 0, PH_LIGHT, PH_HEAVY, PH_PAIRS, PH_NUM };

// CUDA-event spans per phase (only recorded when the context profiles).
struct Prof {
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    struct Span { int phase; cudaEvent_t a, b; };
    std::vector<Span> spans;
    void reset() { used = 0; spans.clear(); }
    cudaEvent_t get() {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    void release() {
        for (auto e : pool) cudaEventDestroy(e);
        pool.clear();
        reset();
    }
};
}  // namespace

struct sspp_ctx {
    sspp_config cfg{};
    std::string err;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
#ifndef SSPP_SIDE_STREAMS
#define SSPP_SIDE_STREAMS 64
#endif
    // CTA-tier launches in flight at once: each holds its stream until its
    // longest chain ends, so a later launch needs a stream of its own
    static constexpr int kSide = SSPP_SIDE_STREAMS;
    cudaStream_t side[kSide] = {};     // heavy-tier launches overlap later light steps and each other
    std::vector<cudaEvent_t> step_ev;  // light step k done
    cudaEvent_t join_ev[kSide] = {};   // side stream joins
    Device D;
    sspp_params params{};          // effective parameters (after autotuning)
    sspp_params user_params{};     // as passed to sspp_init
    int tune_cand = -1;            // autotuner candidate of this run, -1 without autotune
    int tune_shape = 0;            // shape class of the loaded complex (autotuner key)
    bool tune_locked = false;      // a capacity repeat keeps the candidate
    int64_t arena_used = 0;        // arena ints in use after the last reduction
    bool loaded = false, inited = false, computed = false;
    DimInfo hinfo{};
    long long hcounters[CNT_NUM] = {};
    int num_sms = 0;
    int light_blocks_per_sm = 0;
    int heavy_blocks_per_sm = 0;
    int configured_cap1 = -1, configured_cap2 = -1, configured_ht = -1;
    int64_t arena_request = 0;     // ints requested for the arena (grows on CAPACITY)
    int64_t pool_request = 0;      // heavy pool entries requested (grows on CAPACITY)
    double init_ms = 0, compute_ms = 0;
    int64_t ss_steps = 0;
    int* h_err = nullptr;          // pinned
    int* h_gate = nullptr;         // mapped pinned: CTA-tier pool columns finished (mirror)
    int* d_gate = nullptr;         // its device address
    int* h_tail = nullptr;         // pinned: the pool tail after a dimension's sweep
    cudaEvent_t gate_ev = nullptr;
    cudaEvent_t hc_fork = nullptr, hc_join = nullptr;  // guided clearing beside the apparent-pair pass
    long long* h_counters = nullptr;
    unsigned long long* h_dimtot = nullptr;  // pinned: columns per dimension (validation pass)
    DimInfo* h_info = nullptr;
    unsigned long long* h_top = nullptr;
    uint8_t* dropped = nullptr;    // primal reordered numbering (model bit 2)
    int64_t cap_dropped = 0;
    // input buffers owned by the context (host loads); device loads are read in place
    int32_t* own_dims = nullptr;
    int64_t* own_colptr = nullptr;
    int32_t* own_rows = nullptr;
    int64_t cap_own_n = 0, cap_own_nnz = 0;
    int64_t* d_batch = nullptr;    // batch column and entry starts (2 * (k + 1))
    int64_t cap_d_batch = 0;
    Xfer xfer;                     // staged copies from and to caller memory
    HighclearScratch hc;
    CollapseScratch cs;
    BuildScratch bs;               // device complex builders (the input matrix when `built`)
    bool built = false;
    float* bvalues = nullptr;      // a built batch's column values, complex after complex
    int64_t cap_bvalues = 0;
    bool built_batch = false;      // the loaded matrix is a built batch (values in bvalues)
    double build_ms = 0;
    Prof prof;
    double ph_ms[PH_NUM] = {};
    // batch: column range of each complex in the concatenated input, and the
    // sorted pairs copied back once for slicing
    std::vector<int64_t> batch_start;   // k + 1 entries (empty when not a batch)
    std::vector<int64_t> host_pairs;
    bool host_pairs_valid = false;
    std::vector<int64_t> host_ess;     // essentials, copied back once for slicing
    std::vector<int32_t> host_perm;    // reordered -> input index, copied back for representatives
    bool host_perm_valid = false;
    std::vector<int64_t> batch_bounds; // per-complex pair and essential slice starts
    bool host_ess_valid = false;
    int64_t launches = 0, light_launches = 0, heavy_launches = 0;
    // device work queue of (complex, block) items (schedule 2)
    int32_t* q_info = nullptr;     // 3 * k * kNumDims: active counts, min rows, max rows per complex and dimension
    int64_t cap_q_info = 0;
    QItem* q_items = nullptr;
    int64_t cap_q_items = 0;
    int* q_ctr = nullptr;          // taken, done, lin per item
    int64_t cap_q_ctr = 0;
    int32_t* q_cplx = nullptr;     // cur, gate, hpend, item_end, list_cap per complex + 8 scalars
    int64_t cap_q_cplx = 0;
    int64_t* q_loff = nullptr;     // list offsets per complex
    int64_t cap_q_loff = 0;
    int2* q_lists = nullptr;
    int64_t cap_q_lists = 0;
    int32_t* q_pool_c = nullptr;
    int64_t cap_q_pool_c = 0;
    int64_t* q_cstart = nullptr;   // {0, n} when the context holds one complex
    int queue_bpsm = -1;           // queue kernel blocks per SM for q_conf's capacities and threads
    int q_conf[3] = {-1, -1, -1};
    std::vector<int32_t> h_qinfo;
    std::vector<QItem> h_items;
};

namespace {

int set_err(sspp_ctx* c, int code, const std::string& msg) {
    c->err = msg;
    if (c->cfg.verbose) std::fprintf(stderr, "sspp: %s\n", msg.c_str());
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return set_err(ctx, SSPP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

// Device buffers are stream-ordered allocations: growing one neither
// synchronises the device nor waits for other contexts' work, as cudaFree
// would (the server runs several contexts side by side).  Freed memory stays
// in the device's pool for reuse.
template <typename T>
cudaError_t grow(T*& p, int64_t& cap, int64_t want, cudaStream_t s) {
    if (want <= cap && p) return cudaSuccess;
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&p), size_t(std::max<int64_t>(want, 1)) * sizeof(T), s);
    if (e == cudaSuccess) cap = want;
    return e;
}

void free_device(Device& D) {
    void* ptrs[] = {D.dim, D.perm, D.newidx, D.scratch64, D.arena, D.arena_top,
                    D.desc, D.low, D.pivot, D.state, D.cleared, D.negative, D.leftmost, D.active, D.blk, D.dimcnt,
                    D.diminfo, D.err, D.counters, D.step_ctr, D.heavy, D.pool_tail, D.heavy_done, D.death_of, D.pairs,
                    D.ess, D.misc, D.app, D.runlist, D.dimtot};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    D = Device();
}

// Per-column arrays for n columns, input arrays for nnz entries.
int ensure_columns(sspp_ctx* ctx, int64_t n, int64_t nnz) {
    Device& D = ctx->D;
    if (n > INT32_MAX - 8) return set_err(ctx, SSPP_ERR_CAPACITY, "more than 2^31 columns");
    if (n > D.cap_n) {
        int64_t c = n;
        auto g = [&](auto*& p, int64_t mult) {
            using T = std::remove_reference_t<decltype(*p)>;
            int64_t cap = 0;
            if (p) { cudaFreeAsync(p, ctx->stream); p = nullptr; }
            return grow<T>(p, cap, c * mult + 1, ctx->stream);
        };
        CK(g(D.dim, 1));
        CK(g(D.perm, 1));
        CK(g(D.newidx, 1));
        CK(g(D.scratch64, 1));
        CK(g(D.desc, 1));
        CK(g(D.low, 1));
        CK(g(D.pivot, 1));
        CK(g(D.state, 1));
        CK(g(D.cleared, 1));
        CK(g(D.negative, 1));
        CK(g(D.leftmost, 1));
        CK(g(D.active, 1));
        CK(g(D.runlist, 1));
        CK(g(D.death_of, 1));
        CK(g(D.pairs, 2));
        CK(g(D.ess, 1));
        CK(g(D.app, 1));
        D.cap_n = c;
        int64_t nb = (c + 4095) / 4096 + 2;
        CK(grow(D.blk, D.cap_blk, nb, ctx->stream));
        int64_t nbp = (c + 255) / 256 + 1;
        CK(grow(D.dimcnt, D.cap_dimcnt, nbp * kNumDims, ctx->stream));
    }
    if (!D.diminfo) {
        CK(cudaMalloc(&D.diminfo, sizeof(DimInfo)));
        CK(cudaMalloc(&D.err, sizeof(int)));
        CK(cudaMalloc(&D.counters, sizeof(long long) * CNT_NUM));
        CK(cudaMalloc(&D.arena_top, sizeof(unsigned long long)));
        CK(cudaMalloc(&D.pool_tail, sizeof(int)));
        CK(cudaMalloc(&D.heavy_done, sizeof(int)));
        CK(cudaMalloc(&D.misc, sizeof(int64_t) * 8));
        CK(cudaMalloc(&D.dimtot, sizeof(unsigned long long) * kNumDims));
    }
    return SSPP_OK;
}

// Guard ints after the usable arena: staging reads a whole first round of a
// slot (up to 1024 ints) without knowing its length yet.
constexpr int64_t kArenaGuard = 8192;

int ensure_arena(sspp_ctx* ctx, int64_t ints) {
    Device& D = ctx->D;
    if (ints <= D.arena_cap) return SSPP_OK;
    if (D.arena) cudaFreeAsync(D.arena, ctx->stream);
    D.arena = nullptr;
    D.arena_cap = 0;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&D.arena), size_t(ints + kArenaGuard) * sizeof(int32_t), ctx->stream));
    D.arena_cap = ints;
    return SSPP_OK;
}

int64_t arena_need(const sspp_ctx* ctx) {
    const int64_t base = ctx->D.nnz + (kHdr + 3) * ctx->D.n + 4;
    int64_t want = base + std::max<int64_t>(2 * base, int64_t(16) << 20);
    if (ctx->params.dualize || ctx->user_params.autotune == 2) want += base;  // dual columns behind the primal ones
    if (ctx->cfg.arena_bytes > 0) want = std::max<int64_t>(want, ctx->cfg.arena_bytes / 4);
    return std::max(want, ctx->arena_request);
}

// SS schedule of one dimension, following include/specseq.h:603-697.
struct Step {
    int32_t beg, end, minrow;
};

void ss_schedule(const sspp_params& P, int32_t ab, int32_t ae, int32_t minrow_dim, int32_t maxrow_dim,
                 std::vector<Step>& out) {
    if (ae <= ab) return;
    const int kMaxSteps = 4096;
    int64_t ss = std::max(1, P.ss_block_size);
    int32_t b = ab;
    int32_t e = int32_t(std::min<int64_t>(int64_t(ab) + ss, ae));
    int64_t lo = int64_t(maxrow_dim) - ss, hi = lo + ss;
    int steps = 0;
    while ((b < ae || hi > minrow_dim) && steps < kMaxSteps) {
        int32_t mr = int32_t(std::max<int64_t>(lo, INT32_MIN));
        if (e > b) out.push_back({b, e, mr});
        steps++;
        ss = int64_t(float(ss) * P.growth);
        if (ss < 1) ss = 1;
        if (ss > INT32_MAX) ss = INT32_MAX;
        if (hi <= minrow_dim) b = e;
        else { lo -= ss; hi -= ss; }
        if (e < ae) e = int32_t(std::min<int64_t>(int64_t(e) + ss, ae));
    }
    // completion sweep: every remaining column of the dimension, every row
    out.push_back({ab, ae, INT32_MIN});
}

int check_params(sspp_ctx* ctx, const sspp_params* p) {
    if (!p) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null params");
    if (p->dualize < 0 || p->dualize > 2) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dualize must be 0, 1 or 2");
    if (p->model < 0 || p->model > 3) return set_err(ctx, SSPP_ERR_BAD_INPUT, "model must be 0..3");
    if (p->max_iteration < 0) return set_err(ctx, SSPP_ERR_BAD_INPUT, "max_iteration must be >= 0");
    if (p->ss_block_size < 1) return set_err(ctx, SSPP_ERR_BAD_INPUT, "ss_block_size must be >= 1");
    if (!(p->growth >= 1.0f) || !std::isfinite(p->growth))
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "block_size_growth_rate must be >= 1");
    if (p->queue_size < 1) return set_err(ctx, SSPP_ERR_BAD_INPUT, "queue_size must be >= 1");
    if (p->heavy_threads != 0 && p->heavy_threads != 128 && p->heavy_threads != 256)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "heavy_threads must be 0, 128 or 256");
    if (p->level1_capacity < 0 || p->level2_capacity < 0)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "level capacities must be >= 0");
    if (p->autotune < 0 || p->autotune > 2) return set_err(ctx, SSPP_ERR_BAD_INPUT, "autotune must be 0, 1 or 2");
    if (p->representatives < 0 || p->representatives > 1)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "representatives must be 0 or 1");
    if (p->representatives && p->dualize)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "representatives need dualize 0 (the dual reduces cocycles)");
    if (p->schedule < 0 || p->schedule > 2) return set_err(ctx, SSPP_ERR_BAD_INPUT, "schedule must be 0, 1 or 2");
    return SSPP_OK;
}

// autotune 2 may switch to dualization mode 2, which representative cycles rule out
bool tune_allows_dual(const sspp_params& u) { return u.autotune == 2 && !u.representatives; }

// Shared-memory capacities (ints) of the two tiers: a warp holds three
// buffers of level1 ints, a CTA three of level2 ints.
int level1_cap(const sspp_params& p) {
    int c = std::max(32, p.level1_capacity);
    c = std::min(c, 4096);
    return (c + 31) & ~31;
}
int level2_cap(const sspp_params& p) {
    int c = std::max(level1_cap(p), p.level2_capacity);
    c = std::min(c, 18432);
    return (c + 31) & ~31;
}

void span_begin(sspp_ctx* ctx, cudaEvent_t& a, cudaStream_t st = nullptr) {
    if (ctx->cfg.profile) {
        a = ctx->prof.get();
        cudaEventRecord(a, st ? st : ctx->stream);
    }
}
void span_end(sspp_ctx* ctx, int phase, cudaEvent_t a, cudaStream_t st = nullptr) {
    if (ctx->cfg.profile) {
        cudaEvent_t b = ctx->prof.get();
        cudaEventRecord(b, st ? st : ctx->stream);
        ctx->prof.spans.push_back({phase, a, b});
    }
}
// after a stream synchronisation: fold the recorded spans into ph_ms
void span_collect(sspp_ctx* ctx) {
    for (auto& sp : ctx->prof.spans) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) ctx->ph_ms[sp.phase] += ms;
    }
    ctx->prof.reset();
}

// dropped[] of the edge collapse when it runs (model bit 2), else null
const uint8_t* dropped_of(const sspp_ctx* ctx) { return (ctx->params.model & 2) ? ctx->dropped : nullptr; }

// Edge collapse on the reordered matrix (needs host reads of the column
// ranges, the edge count and the largest degree).
int run_collapse(sspp_ctx* ctx) {
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    if (D.n > ctx->cap_dropped) {
        if (ctx->dropped) cudaFreeAsync(ctx->dropped, s);
        ctx->dropped = nullptr;
        ctx->cap_dropped = 0;
        CK(grow(ctx->dropped, ctx->cap_dropped, D.n, s));
    }
    CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const DimInfo info = *ctx->h_info;
    const char* msg = nullptr;
    const int k = collapse(D, info, ctx->dropped, ctx->cs, s, &msg);
    if (k < 0) return set_err(ctx, SSPP_ERR_CUDA, msg ? msg : "edge collapse failed");
    ctx->launches += k;
    CK(cudaGetLastError());
    return SSPP_OK;
}

// Reordered column ranges of the dimensions from the validation pass's counts
// (the reorder groups columns by ascending dimension, stably).
DimInfo ranges_of_counts(const unsigned long long* cnt) {
    DimInfo r{};
    int64_t s = 0;
    for (int d = 0; d < kNumDims; d++) {
        r.col_begin[d] = int32_t(s);
        s += int64_t(cnt[d]);
        r.col_end[d] = int32_t(s);
    }
    return r;
}

// Sizes the guided-clearing scratch from the per-dimension column ranges and
// runs it on stream `s`.  `ranges` gives the ranges; without it they are read
// back through the context's stream, whose work so far (the reorder) they
// come from.
int run_highclear(sspp_ctx* ctx, cudaStream_t s, const DimInfo* ranges = nullptr, bool from_input = false) {
    Device& D = ctx->D;
    DimInfo info;
    if (ranges) {
        info = *ranges;
    } else {
        CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        info = *ctx->h_info;
    }
    HighclearScratch& S = ctx->hc;
    int top = -1;
    for (int d = kMaxDim; d >= 1; d--)
        if (info.col_end[d] > info.col_begin[d]) { top = d; break; }
    if (top < 1) return SSPP_OK;
    for (int d = 1; d <= top; d++)
        CK(grow(S.tup[d], S.cap_tup[d], int64_t(d + 1) * (info.col_end[d] - info.col_begin[d]) + 1, s));
    const int64_t nv = info.col_end[0] - info.col_begin[0];
    const int64_t ne = info.col_end[1] - info.col_begin[1];
    CK(grow(S.deg, S.cap_deg, nv + 2, s));
    CK(grow(S.blk, S.cap_blk, (nv + 1) / 4096 + 4, s));  // scan block sums (4,096 per block)
    CK(grow(S.adj_off, S.cap_adj_off, nv + 2, s));
    CK(grow(S.adj, S.cap_adj, 2 * ne + 1, s));
    if (ctx->params.max_iteration <= kMaskCandidates) {
        CK(grow(S.adj_src, S.cap_src, 2 * ne + 1, s));
        CK(grow(S.nmask, S.cap_nmask, 2 * ne + 1, s));
    }
    const int64_t ntop = info.col_end[top] - info.col_begin[top];
    int64_t slots = 1024;
    while (slots < 2 * ntop) slots *= 2;
    CK(grow(S.table, S.cap_table, slots, s));
    S.mask = uint32_t(slots - 1);
    ctx->launches += highclear(D, info, ctx->params.max_iteration, dropped_of(ctx), S, s, from_input);
    return SSPP_OK;
}

// Autotuned parameters for the loaded complex, chosen once its dimension
// ranges are known (one host read): the shape key is the top dimension and
// the quarter of the columns that lie in it.
int autotune_choose(sspp_ctx* ctx) {
    Device& D = ctx->D;
    CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const DimInfo& I = *ctx->h_info;
    int top = 0;
    for (int d = kMaxDim; d >= 0; d--)
        if (I.col_end[d] > I.col_begin[d]) { top = d; break; }
    const double frac = D.n ? double(I.col_end[top] - I.col_begin[top]) / double(D.n) : 0.0;
    ctx->tune_shape = top * 4 + std::min(3, int(frac * 4.0));
    const sspp_params& u = ctx->user_params;
    Knobs k;
    // contexts that share the GPU (a server's workers) do not try candidates on large inputs
    ctx->tune_cand = tune_choose(D.n, ctx->tune_shape, u.model, u.dualize, tune_allows_dual(u), &k,
                                 ctx->cfg.sm_share <= 1);
    sspp_params& q = ctx->params;
    q.ss_block_size = k.ss_block_size;
    q.growth = k.growth;
    q.queue_size = k.queue_size;
    q.level1_capacity = k.level1;
    q.level2_capacity = k.level2;
    q.heavy_threads = k.heavy_threads;
    q.dualize = k.dualize;
    return SSPP_OK;
}

int run_init(sspp_ctx* ctx) {
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    ctx->prof.reset();
    for (double& x : ctx->ph_ms) x = 0;
    ctx->launches = ctx->light_launches = ctx->heavy_launches = 0;
    CK(cudaMemsetAsync(D.err, 0, sizeof(int), s));
    CK(cudaMemsetAsync(D.counters, 0, sizeof(long long) * CNT_NUM, s));
    int rc = ensure_arena(ctx, arena_need(ctx));
    if (rc) return rc;
    if (D.n == 0) {  // nothing to reduce
        std::memset(&ctx->hinfo, 0, sizeof(ctx->hinfo));
        std::memset(ctx->hcounters, 0, sizeof(ctx->hcounters));
        ctx->init_ms = 0;
        ctx->inited = true;
        ctx->computed = false;
        return SSPP_OK;
    }
    cudaEvent_t ev0 = nullptr;
    span_begin(ctx, ev0);
    ctx->launches += validate(D, s);
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_dimtot, D.dimtot, sizeof(unsigned long long) * kNumDims, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*ctx->h_err) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dimension out of range 0..7 or malformed col_ptr");
    const DimInfo ranges = ranges_of_counts(ctx->h_dimtot);
    // the reorder also does the first init pass unless an edge collapse will
    // empty columns in between (the autotuner never changes the model)
    const bool lows_in_reorder = !(ctx->params.model & 2);
    // guided clearing reads only the matrix and marks top-dimension columns,
    // the apparent-pair pass marks youngest facets (never of the top
    // dimension): the two run side by side and the compression waits for both.
    // Without an edge collapse guided clearing starts as soon as the reorder
    // has assigned the new indices (its tuples come from the input columns).
    const bool guided = (ctx->params.model & 1) && ctx->params.max_iteration > 0;
    const bool early = guided && !(ctx->params.model & 2);
    ctx->launches += reorder(D, lows_in_reorder, s, early ? ctx->hc_fork : nullptr);
    CK(cudaMemcpyAsync(D.arena_top, D.blk + reorder_total_slot(D), sizeof(unsigned long long),
                       cudaMemcpyDeviceToDevice, s));
    if (ctx->user_params.autotune && !ctx->tune_locked) {
        int rc2 = autotune_choose(ctx);
        if (rc2) return rc2;
    }
    if (ctx->params.model & 2) {  // collapse before everything else: dropped columns are emptied
        int rc2 = run_collapse(ctx);
        if (rc2) return rc2;
    }
    if (guided) {
        cudaStream_t hs = ctx->side[0];
        if (!early) CK(cudaEventRecord(ctx->hc_fork, s));  // after the collapse
        CK(cudaStreamWaitEvent(hs, ctx->hc_fork, 0));
        int rc2 = run_highclear(ctx, hs, &ranges, early);
        CK(cudaEventRecord(ctx->hc_join, hs));
        if (rc2) {
            CK(cudaStreamWaitEvent(s, ctx->hc_join, 0));
            return rc2;
        }
    }
    ctx->launches += init_passes(D, lows_in_reorder, s);
    if (guided) CK(cudaStreamWaitEvent(s, ctx->hc_join, 0));
    ctx->launches += init_compress(D, dropped_of(ctx), ctx->params.representatives != 0, ctx->params.dualize != 1, s);
    if (ctx->params.dualize == 1) {
        ctx->launches += dualize(D, 1, s);
        ctx->launches += build_apparent(D, s);
    }
    ctx->launches += active_list(D, ctx->params.dualize != 1, s);
    span_end(ctx, PH_INIT, ev0);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_counters, D.counters, sizeof(long long) * CNT_NUM, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->hinfo = *ctx->h_info;
    std::memcpy(ctx->hcounters, ctx->h_counters, sizeof(ctx->hcounters));
    ctx->init_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    span_collect(ctx);
    if (*ctx->h_err & ERRB_BAD_INPUT)
        return set_err(ctx, SSPP_ERR_BAD_INPUT,
                       "malformed boundary matrix (a face index out of range, unsorted, duplicated, or of the "
                       "wrong dimension)");
    if (*ctx->h_err & ERRB_CHECK) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dualization self-check failed");
    if (*ctx->h_err) return set_err(ctx, SSPP_ERR_CAPACITY, "init pass overflow");
    ctx->inited = true;
    ctx->computed = false;
    return SSPP_OK;
}

// Runs one spectral-sequence schedule: per step a light-tier launch on the
// main stream and a heavy-tier launch for the columns it deferred.
// Dimension gate.  The next dimension's columns are cleared by the claims of
// this one, so it used to start only once every CTA-tier column of this
// dimension was done; on large grids the last few of them are single long
// chains that leave the GPU idle for milliseconds.  Instead the host waits
// (after the sweep, which leaves only CTA-tier columns) until at most
// kGateLeft pool columns are unfinished, then goes on.  A column of the next
// dimension reduced before its row is cleared is a positive column: it
// reduces to zero, or any row it claims is taken back by the smaller column
// whose reduced lowest row it is (the pivots of a reduced matrix are unique),
// so the pairs do not change; only that column's work is wasted, and at most
// kGateLeft rows can be cleared late.  Progress comes from the CTA tier's
// mirror in mapped host memory (a lower bound); the wait also ends when every
// side stream is idle, or after kGateMaxMs.  The polling thread yields its core
// between reads, and after kGateSpinMs of waiting sleeps kGateNapUs between
// them, so a server's workers do not each hold a spinning core.
constexpr int64_t kGateMinCols = int64_t(1) << 17;
constexpr int kGateLeft = 16;
constexpr double kGateMaxMs = 30000.0;
constexpr double kGateSpinMs = 2.0;
constexpr int kGateNapUs = 50;

int dimension_gate(sspp_ctx* ctx) {
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->h_tail, ctx->D.pool_tail, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ctx->gate_ev, s));
    CK(cudaEventSynchronize(ctx->gate_ev));
    const int tail = *ctx->h_tail;
    const auto t0 = std::chrono::steady_clock::now();
    for (int it = 1;; it++) {
        const int done = *reinterpret_cast<volatile int*>(ctx->h_gate);
        if (tail - done <= kGateLeft) break;
        if ((it & 63) == 0) {
            bool idle = true;
            for (int q = 0; q < sspp_ctx::kSide && idle; q++) idle = cudaStreamQuery(ctx->side[q]) != cudaErrorNotReady;
            if (idle) break;
            const double waited =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (waited > kGateMaxMs) break;
            if (waited > kGateSpinMs) {
                std::this_thread::sleep_for(std::chrono::microseconds(kGateNapUs));
                continue;
            }
        }
        std::this_thread::yield();
    }
    return SSPP_OK;
}

constexpr int kStepCtr = 8;  // counters per spectral-sequence step (see ReduceArgs::ctr)

int run_steps(sspp_ctx* ctx, const std::vector<Step>& steps, int cap1, int cap2, int ht) {
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    const sspp_params& P = ctx->params;
    if (kStepCtr * int64_t(steps.size()) > D.cap_steps) {
        if (D.step_ctr) cudaFreeAsync(D.step_ctr, s);
        D.step_ctr = nullptr;
        D.cap_steps = 0;
        CK(grow(D.step_ctr, D.cap_steps, kStepCtr * int64_t(steps.size()) + 64, s));
    }
    if (!steps.empty()) CK(cudaMemsetAsync(D.step_ctr, 0, sizeof(int) * kStepCtr * steps.size(), s));
    // heavy pool: deferrals are rare (heavy columns and displaced owners); a
    // full pool sets the capacity bit and the run is repeated with a larger one
    const int64_t want_pool = std::max<int64_t>(ctx->pool_request, std::max<int64_t>(D.n / 4, 1 << 16));
    if (want_pool > D.pool_cap) {
        if (D.heavy) cudaFreeAsync(D.heavy, s);
        D.heavy = nullptr;
        D.pool_cap = 0;
        CK(grow(D.heavy, D.pool_cap, want_pool, s));
    }
    CK(cudaMemsetAsync(D.pool_tail, 0, sizeof(int), s));
    const int light_max = std::max(1, ctx->num_sms * ctx->light_blocks_per_sm);
    const int heavy_grid = std::max(1, std::min(ctx->num_sms * ctx->heavy_blocks_per_sm, 2 * ctx->num_sms));
    const int q_blocks = std::max(1, (P.queue_size + 3) / 4);
#ifndef SSPP_LIGHT_CHUNK
#define SSPP_LIGHT_CHUNK 8
#endif
#ifndef SSPP_LIGHT_FILTER
#define SSPP_LIGHT_FILTER 1
#endif
#ifndef SSPP_FILTER_CHUNK
#define SSPP_FILTER_CHUNK 1
#endif
    // Each step first lists its runnable columns (k_light_filter, one thread
    // per window entry), then warps take them SSPP_FILTER_CHUNK at a time;
    // without the filter, warps walk the window SSPP_LIGHT_CHUNK entries at a
    // time through one shared counter.
    const bool filtered = SSPP_LIGHT_FILTER != 0;
    const int chunk = filtered ? SSPP_FILTER_CHUNK : SSPP_LIGHT_CHUNK;
    // Heavy launches go to side streams (round robin) after their light step:
    // they overlap the following light steps and each other, so long chains of
    // different steps run concurrently.  Each dimension's completion sweep, and
    // the next dimension, wait for all of them (twist clearing needs the
    // finished dimension) -- on large inputs only until few of them are left
    // (the dimension gate below).
    const bool overlap = true;
    const bool gate = D.n >= kGateMinCols && ctx->h_gate && ctx->d_gate && ctx->h_tail && ctx->gate_ev;
    D.gate_host = gate ? ctx->d_gate : nullptr;
    if (gate) {
        *reinterpret_cast<volatile int*>(ctx->h_gate) = 0;  // no CTA-tier launch of this context is running
        CK(cudaMemsetAsync(D.heavy_done, 0, sizeof(int), s));
    }
    while (ctx->step_ev.size() < steps.size() + 1) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        ctx->step_ev.push_back(ev);
    }
    auto join_sides = [&]() -> int {
        for (int q = 0; q < sspp_ctx::kSide; q++) {
            CK(cudaEventRecord(ctx->join_ev[q], ctx->side[q]));
            CK(cudaStreamWaitEvent(s, ctx->join_ev[q], 0));
        }
        return SSPP_OK;
    };
    for (size_t k = 0; k < steps.size(); k++) {
        const Step& st = steps[k];
        const bool last_of_dim = st.minrow == INT32_MIN;
        if (overlap && last_of_dim && !gate) {  // join: everything heavy of this dimension is done
            int rcj = join_sides();
            if (rcj) return rcj;
        }
        int64_t chunks = (int64_t(st.end - st.beg) + chunk - 1) / chunk;
        int grid = int(std::min<int64_t>(std::min<int64_t>((chunks + 3) / 4, light_max), q_blocks));
        grid = std::max(grid, 1);
        int* ctr = D.step_ctr + kStepCtr * k;
        cudaEvent_t a = nullptr, b = nullptr;
        span_begin(ctx, a);
        int* ctr_next = k + 1 < steps.size() ? ctr + kStepCtr : nullptr;
        if (filtered) {
            const int fgrid = int(std::max<int64_t>(
                1, std::min<int64_t>((int64_t(st.end - st.beg) + 255) / 256, int64_t(ctx->num_sms) * 8)));
            reduce_light_filtered_launch(D, st.beg, st.end, st.minrow, cap1, chunk, ctr, ctr_next, fgrid, grid, s);
            ctx->launches++;
        } else {
            reduce_light_launch(D, D.active, st.beg, st.end, st.minrow, cap1, chunk, ctr, ctr_next, grid, s);
        }
        span_end(ctx, PH_LIGHT, a);
        if (overlap && (!last_of_dim || gate)) {
            // an idle side stream if there is one: a CTA-tier launch lasts as
            // long as its longest chain, and a launch queued behind it on the
            // same stream would wait for that chain
            int q = int(k % sspp_ctx::kSide);
#ifndef SSPP_SIDE_RR
            for (int t = 0; t < sspp_ctx::kSide; t++) {
                const int c = int((k + t) % sspp_ctx::kSide);
                if (cudaStreamQuery(ctx->side[c]) == cudaSuccess) {
                    q = c;
                    break;
                }
            }
#endif
            cudaStream_t hs = ctx->side[q];
            CK(cudaEventRecord(ctx->step_ev[k], s));
            CK(cudaStreamWaitEvent(hs, ctx->step_ev[k], 0));
            span_begin(ctx, b, hs);
            reduce_heavy_launch(D, cap2, ht, ctr, heavy_grid, hs);
            span_end(ctx, PH_HEAVY, b, hs);
        } else {
            span_begin(ctx, b);
            reduce_heavy_launch(D, cap2, ht, ctr, heavy_grid, s);
            span_end(ctx, PH_HEAVY, b);
        }
        ctx->light_launches++;
        ctx->heavy_launches++;
        ctx->launches += 2;
        if (gate && last_of_dim && k + 1 < steps.size()) {
            int rcg = dimension_gate(ctx);
            if (rcg) return rcg;
        }
    }
    if (overlap) {  // nothing may still run on a side stream past this point
        int rcj = join_sides();
        if (rcj) return rcj;
    }
    ctx->ss_steps = int64_t(steps.size());
    return SSPP_OK;
}

// Spectral-sequence blocks of dimensions [dlo, dhi] (ascending or
// descending) of every complex the context holds, as one persistent launch
// draining a device queue of (complex, block) items (k_reduce_queue).  Each
// complex gets the schedule ss_schedule gives its own active columns and row
// bounds; the host reads those per-complex bounds once (one synchronisation)
// and issues one launch.
constexpr int kQueueChunk = 8;
constexpr int kQueueGateLeft = 16;

int run_queue(sspp_ctx* ctx, int dlo, int dhi, bool ascending, int cap1, int cap2, int threads) {
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    const sspp_params& P = ctx->params;
    const bool batch = ctx->batch_start.size() >= 2;
    const int32_t k = batch ? int32_t(ctx->batch_start.size() - 1) : 1;
    const int64_t* d_cstart = ctx->d_batch;
    if (!batch) {
        if (!ctx->q_cstart) CK(cudaMalloc(&ctx->q_cstart, 2 * sizeof(int64_t)));
        const int64_t h[2] = {0, D.n};
        CK(cudaMemcpyAsync(ctx->q_cstart, h, sizeof(h), cudaMemcpyHostToDevice, s));
        d_cstart = ctx->q_cstart;
    }
    const int64_t m = int64_t(k) * kNumDims;
    CK(grow(ctx->q_info, ctx->cap_q_info, 3 * m, s));
    ctx->launches += queue_complex_info(D, k, d_cstart, ctx->q_info, ctx->q_info + m, ctx->q_info + 2 * m, s);
    ctx->h_qinfo.resize(size_t(3 * m));
    CK(cudaMemcpyAsync(ctx->h_qinfo.data(), ctx->q_info, sizeof(int32_t) * 3 * m, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int32_t* act = ctx->h_qinfo.data();
    const int32_t* mnr = act + m;
    const int32_t* mxr = act + 2 * m;
    const DimInfo& I = ctx->hinfo;
    // items, complex by complex; the active list holds each dimension's
    // columns complex after complex
    std::vector<QItem>& items = ctx->h_items;
    items.clear();
    const size_t nk = size_t(k);
    std::vector<int32_t> first(nk, 0), iend(nk, 0), lcap(nk, 0);
    std::vector<int64_t> loff(nk + 1, 0);
    std::vector<int32_t> dim_start(kNumDims);
    for (int d = 0; d < kNumDims; d++) dim_start[d] = I.act_begin[d];
    std::vector<Step> st;
    for (int32_t c = 0; c < k; c++) {
        first[size_t(c)] = int32_t(items.size());
        int32_t cap = 0;
        for (int j = 0; j <= dhi - dlo; j++) {
            const int d = ascending ? dlo + j : dhi - j;
            const int32_t cnt = act[int64_t(c) * kNumDims + d];
            const int32_t ab = dim_start[d], ae = ab + cnt;
            cap = std::max(cap, cnt);
            st.clear();
            const int32_t mr = mnr[int64_t(c) * kNumDims + d];
            ss_schedule(P, ab, ae, mr == INT32_MAX ? 0 : mr, mxr[int64_t(c) * kNumDims + d], st);
            int32_t eprev = -1;
            const size_t d0 = items.size();
            for (const Step& x : st) {
                QItem q{};
                q.cplx = c;
                q.nbeg = eprev < 0 ? x.beg : std::max(eprev, x.beg);
                q.nend = std::max(q.nbeg, x.end);
                eprev = std::max(eprev, x.end);
                q.minrow = x.minrow;
                q.flags = ((items.size() - d0) & 1) ? QF_HALF : 0;
                items.push_back(q);
            }
            if (items.size() > d0) items.back().flags |= QF_LAST_OF_DIM;
        }
        // dimensions outside [dlo, dhi] keep their columns, but the running
        // offsets cover every dimension
        for (int d = 0; d < kNumDims; d++) dim_start[d] += act[int64_t(c) * kNumDims + d];
        iend[size_t(c)] = int32_t(items.size());
        lcap[size_t(c)] = cap + 32;
        loff[size_t(c) + 1] = loff[size_t(c)] + 2 * int64_t(lcap[size_t(c)]);
    }
    const int64_t nit = int64_t(items.size());
    ctx->ss_steps = nit;
    if (nit == 0) return SSPP_OK;
    if (ctx->queue_bpsm < 0 || cap1 != ctx->q_conf[0] || cap2 != ctx->q_conf[1] || threads != ctx->q_conf[2]) {
        int b = 0;
        CK(queue_configure(cap1, cap2, threads, &b));
        ctx->queue_bpsm = b;
        ctx->q_conf[0] = cap1;
        ctx->q_conf[1] = cap2;
        ctx->q_conf[2] = threads;
    }
    if (ctx->queue_bpsm < 1) return set_err(ctx, SSPP_ERR_CAPACITY, "level capacities too large for shared memory");
    // device state
    CK(grow(ctx->q_items, ctx->cap_q_items, nit, s));
    CK(grow(ctx->q_ctr, ctx->cap_q_ctr, 3 * (nit + 1), s));
    CK(grow(ctx->q_cplx, ctx->cap_q_cplx, 5 * int64_t(k) + 8, s));
    CK(grow(ctx->q_loff, ctx->cap_q_loff, int64_t(k), s));
    CK(grow(ctx->q_lists, ctx->cap_q_lists, std::max<int64_t>(loff[size_t(k)], 1), s));
    const int64_t want_pool = std::max<int64_t>(ctx->pool_request, std::max<int64_t>(D.n / 4, 1 << 16));
    if (want_pool > D.pool_cap) {
        if (D.heavy) cudaFreeAsync(D.heavy, s);
        D.heavy = nullptr;
        D.pool_cap = 0;
        CK(grow(D.heavy, D.pool_cap, want_pool, s));
    }
    if (D.pool_cap > ctx->cap_q_pool_c) {
        if (ctx->q_pool_c) cudaFreeAsync(ctx->q_pool_c, s);
        ctx->q_pool_c = nullptr;
        ctx->cap_q_pool_c = 0;
        CK(grow(ctx->q_pool_c, ctx->cap_q_pool_c, D.pool_cap, s));
    }
    std::vector<int32_t> hc(size_t(5 * int64_t(k) + 8), 0);
    int32_t nfin = 0;
    for (int32_t c = 0; c < k; c++) {
        const bool none = first[size_t(c)] == iend[size_t(c)];
        hc[size_t(c)] = none ? -1 : first[size_t(c)];   // cur
        nfin += none ? 1 : 0;
        hc[size_t(3 * k + c)] = iend[size_t(c)];         // item_end
        hc[size_t(4 * k + c)] = lcap[size_t(c)];         // list_cap
    }
    hc[size_t(5 * k)] = nfin;  // finished; then abort, pool_head, pool_tail
    CK(cudaMemcpyAsync(ctx->q_items, items.data(), sizeof(QItem) * size_t(nit), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->q_cplx, hc.data(), sizeof(int32_t) * hc.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->q_loff, loff.data(), sizeof(int64_t) * size_t(k), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->q_ctr, 0, sizeof(int) * 3 * size_t(nit + 1), s));
    CK(cudaMemsetAsync(D.heavy, 0xff, sizeof(int32_t) * size_t(D.pool_cap), s));
    QueueArgs Q{};
    Q.items = ctx->q_items;
    Q.nitems = int32_t(nit);
    Q.ncplx = k;
    Q.taken = ctx->q_ctr;
    Q.done = ctx->q_ctr + (nit + 1);
    Q.lin = ctx->q_ctr + 2 * (nit + 1);
    Q.cur = ctx->q_cplx;
    Q.gate = ctx->q_cplx + k;
    Q.hpend = ctx->q_cplx + 2 * k;
    Q.item_end = ctx->q_cplx + 3 * k;
    Q.list_cap = ctx->q_cplx + 4 * k;
    Q.finished = ctx->q_cplx + 5 * k;
    Q.abort = ctx->q_cplx + 5 * k + 1;
    Q.pool_head = ctx->q_cplx + 5 * k + 2;
    Q.pool_tail = ctx->q_cplx + 5 * k + 3;
    Q.list_off = ctx->q_loff;
    Q.lists = ctx->q_lists;
    Q.pool = D.heavy;
    Q.pool_c = ctx->q_pool_c;
    Q.pool_cap = int32_t(std::min<int64_t>(D.pool_cap, INT32_MAX));
    Q.gate_left = kQueueGateLeft;
    Q.chunk = kQueueChunk;
    Q.cap1 = cap1;
    Q.spin_limit = (long long)1 << 22;  // idle polls of about a quarter to one microsecond each
    const int share = std::max(1, ctx->cfg.sm_share);
    const int sms = std::max(1, ctx->num_sms / share);
    const int grid = std::max(2, sms * ctx->queue_bpsm);
    // a block per SM for the CTA tier (half the blocks when only one fits per SM)
    Q.heavy_ctas = ctx->queue_bpsm >= 2 ? sms : std::max(1, grid / 2);
    cudaEvent_t a = nullptr;
    span_begin(ctx, a);
    CK(reduce_queue_launch(D, cap1, cap2, threads, Q, grid, s));
    span_end(ctx, PH_LIGHT, a);
    ctx->launches += 1;
    ctx->light_launches += 1;
    return SSPP_OK;
}

int run_compute(sspp_ctx* ctx) {
    ctx->err.clear();
    ctx->host_pairs_valid = false;
    ctx->host_ess_valid = false;
    ctx->host_perm_valid = false;
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    if (D.n == 0) {
        std::memset(ctx->hcounters, 0, sizeof(ctx->hcounters));
        ctx->compute_ms = 0;
        ctx->ss_steps = 0;
        ctx->computed = true;
        return SSPP_OK;
    }
    const sspp_params& P = ctx->params;
    const int cap1 = level1_cap(P), cap2 = level2_cap(P);
    const int ht = P.heavy_threads == 128 ? 128 : 256;
    if (cap1 != ctx->configured_cap1 || cap2 != ctx->configured_cap2 || ht != ctx->configured_ht) {
        CK(reduce_configure(cap1, cap2, ht, &ctx->light_blocks_per_sm, &ctx->heavy_blocks_per_sm));
        ctx->configured_cap1 = cap1;
        ctx->configured_cap2 = cap2;
        ctx->configured_ht = ht;
        if (ctx->light_blocks_per_sm < 1 || ctx->heavy_blocks_per_sm < 1)
            return set_err(ctx, SSPP_ERR_CAPACITY, "level capacities too large for shared memory");
    }
    // schedule: dimensions high to low, or low to high for the dual matrix
    // (include/specseq.h:598-600).  dualize 2: the boundary matrix's edge
    // columns first (0-dimensional pairs), then the coboundary matrix from
    // dimension 1 up.
    const DimInfo& I = ctx->hinfo;
    auto schedule = [&](int dlo, int dhi, bool ascending) {
        std::vector<Step> st;
        for (int k = 0; k <= dhi - dlo; k++) {
            const int d = ascending ? dlo + k : dhi - k;
            ss_schedule(P, I.act_begin[d], I.act_end[d], I.min_row[d] == INT_MAX ? 0 : I.min_row[d], I.max_row[d], st);
        }
        return st;
    };
    // schedule 1 (and 0): a host loop of per-block launches; 2: one persistent
    // launch per phase draining the (complex, block) work queue.  The host loop
    // is the default: its warp-tier kernel keeps four times as many warps
    // resident as the persistent kernel, whose CTA-tier role sets the register
    // budget of every block
    const bool queue = P.schedule == 2;
    auto phase = [&](int dlo, int dhi, bool ascending) {
        return queue ? run_queue(ctx, dlo, dhi, ascending, cap1, cap2, ht)
                     : run_steps(ctx, schedule(dlo, dhi, ascending), cap1, cap2, ht);
    };
    int64_t nsteps = 0;
    if (P.dualize == 2) {
        int rc = phase(1, 1, false);
        if (rc) return rc;
        nsteps += ctx->ss_steps;
        ctx->launches += dualize(D, 2, s);
        ctx->launches += build_apparent(D, s);
        ctx->launches += active_list(D, false, s);
        CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        ctx->hinfo = *ctx->h_info;
        rc = phase(1, kMaxDim, true);
        if (rc) return rc;
        nsteps += ctx->ss_steps;
    } else {
        int rc = P.dualize ? phase(0, kMaxDim, true) : phase(0, kMaxDim, false);
        if (rc) return rc;
        nsteps += ctx->ss_steps;
    }
    ctx->ss_steps = nsteps;
    cudaEvent_t ep = nullptr;
    span_begin(ctx, ep);
    ctx->launches += extract_pairs(D, P.dualize != 0, dropped_of(ctx), s);
    span_end(ctx, PH_PAIRS, ep);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_counters, D.counters, sizeof(long long) * CNT_NUM, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_top, D.arena_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::memcpy(ctx->hcounters, ctx->h_counters, sizeof(ctx->hcounters));
    ctx->arena_used = int64_t(*ctx->h_top);
    ctx->compute_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    span_collect(ctx);
    const int e = *ctx->h_err;
    if (e & ERRB_CAPACITY) return SSPP_ERR_CAPACITY;
    if (e & ERRB_LEN) return set_err(ctx, SSPP_ERR_CAPACITY, "a column exceeded 2^24 entries");
    if (e & ERRB_TIMEOUT) return set_err(ctx, SSPP_ERR_TIMEOUT, "per-column merge limit reached");
    if (e & ERRB_CHECK) return set_err(ctx, SSPP_ERR_BAD_INPUT, "reduction self-check failed (bad index skipped)");
    if (e) return set_err(ctx, SSPP_ERR_BAD_INPUT, "device error word set");
    ctx->computed = true;
    return SSPP_OK;
}

int load_common(sspp_ctx* ctx, int64_t n, int64_t nnz) {
    ctx->loaded = ctx->inited = ctx->computed = false;
    ctx->built = false;
    ctx->built_batch = false;
    ctx->build_ms = 0;
    ctx->batch_start.clear();
    ctx->host_pairs_valid = false;
    ctx->host_ess_valid = false;
    int rc = ensure_columns(ctx, std::max<int64_t>(n, 1), std::max<int64_t>(nnz, 1));
    if (rc) return rc;
    ctx->D.n = n;
    ctx->D.nnz = nnz;
    ctx->arena_request = 0;
    return SSPP_OK;
}

// Device buffers for inputs copied from the host (grown, never shrunk).
int ensure_own(sspp_ctx* ctx, int64_t n, int64_t nnz) {
    if (n + 1 > ctx->cap_own_n) {
        if (ctx->own_dims) cudaFreeAsync(ctx->own_dims, ctx->stream);
        if (ctx->own_colptr) cudaFreeAsync(ctx->own_colptr, ctx->stream);
        ctx->own_dims = nullptr;
        ctx->own_colptr = nullptr;
        ctx->cap_own_n = 0;
        int64_t c1 = 0, c2 = 0;
        CK(grow(ctx->own_dims, c1, n + 1, ctx->stream));
        CK(grow(ctx->own_colptr, c2, n + 1, ctx->stream));
        ctx->cap_own_n = n + 1;
    }
    if (nnz > ctx->cap_own_nnz || !ctx->own_rows) {
        if (ctx->own_rows) cudaFreeAsync(ctx->own_rows, ctx->stream);
        ctx->own_rows = nullptr;
        ctx->cap_own_nnz = 0;
        int64_t c3 = 0;
        CK(grow(ctx->own_rows, c3, std::max<int64_t>(nnz, 1), ctx->stream));
        ctx->cap_own_nnz = std::max<int64_t>(nnz, 1);
    }
    return SSPP_OK;
}

// A device pointer to `count` floats of the caller: the pointer itself when it
// is device (or managed) memory of this context's device, else a copy in the
// builder's input buffer.
int stage_floats(sspp_ctx* ctx, const float* p, int64_t count, const float** out) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        a.type = cudaMemoryTypeUnregistered;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) {
        if (a.type == cudaMemoryTypeDevice && a.device != ctx->cfg.device)
            return set_err(ctx, SSPP_ERR_BAD_INPUT, "input is in another device's memory");
        *out = p;
        return SSPP_OK;
    }
    void* d = nullptr;
    const size_t bytes = sizeof(float) * size_t(count);
    CK(build_stage(ctx->bs, bytes, ctx->stream, &d));
    CK(ctx->xfer.h2d({{p, d, bytes}}, ctx->stream));
    *out = static_cast<const float*>(d);
    return SSPP_OK;
}

int finish_build(sspp_ctx* ctx, int rc, const Built& b, const std::string& msg,
                 std::chrono::steady_clock::time_point t0) {
    if (rc) return set_err(ctx, rc == -1 ? SSPP_ERR_BAD_INPUT : SSPP_ERR_CUDA, msg);
    rc = load_common(ctx, b.ncols, b.nnz);
    if (rc) return rc;
    ctx->D.in_dims = b.dims;
    ctx->D.in_colptr = b.col_ptr;
    ctx->D.in_rows = b.rows;
    ctx->loaded = true;
    ctx->built = true;
    ctx->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SSPP_OK;
}

}  // namespace

namespace {

// A device buffer of `want` T that keeps its first `used` entries.
template <typename T>
cudaError_t grow_keep(T*& p, int64_t& cap, int64_t want, int64_t used, cudaStream_t s) {
    if (want <= cap && p) return cudaSuccess;
    const int64_t nc = std::max<int64_t>(want, cap + cap / 2);
    T* q = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&q), size_t(std::max<int64_t>(nc, 1)) * sizeof(T), s);
    if (e != cudaSuccess) return e;
    if (p && used > 0) e = cudaMemcpyAsync(q, p, size_t(used) * sizeof(T), cudaMemcpyDeviceToDevice, s);
    if (p) cudaFreeAsync(p, s);
    p = q;
    cap = nc;
    return e;
}

// own_dims and own_colptr share one capacity (cap_own_n); they keep their
// first `used` and `used + 1` entries
cudaError_t grow_own_cols(sspp_ctx* ctx, int64_t want, int64_t used, cudaStream_t s) {
    if (want <= ctx->cap_own_n && ctx->own_dims && ctx->own_colptr) return cudaSuccess;
    int64_t c1 = ctx->own_dims ? ctx->cap_own_n : 0, c2 = ctx->own_colptr ? ctx->cap_own_n : 0;
    cudaError_t e = grow_keep(ctx->own_dims, c1, want, used, s);
    if (e == cudaSuccess) e = grow_keep(ctx->own_colptr, c2, c1, used + 1, s);
    ctx->cap_own_n = std::min(c1, c2);
    return e;
}

}  // namespace

extern "C" {

void sspp_default_params(sspp_params* p) {
    if (!p) return;
    p->dualize = 0;
    p->representatives = 0;
    p->model = 0;
    p->max_iteration = 0;
    p->ss_block_size = 102400;
    p->growth = 1.05f;
    p->queue_size = 65536;
    p->level1_capacity = 1000;
    p->level2_capacity = 8000;
    p->autotune = 0;
    p->heavy_threads = 0;
    p->schedule = 0;
}

sspp_ctx* sspp_create(const sspp_config* cfg) {
    auto* ctx = new (std::nothrow) sspp_ctx;
    if (!ctx) return nullptr;
    if (cfg) ctx->cfg = *cfg;
    ctx->xfer.set_threads(ctx->cfg.host_threads);
    if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) { delete ctx; return nullptr; }
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return nullptr; }
    for (int q = 0; q < sspp_ctx::kSide; q++) {
        if (cudaStreamCreateWithFlags(&ctx->side[q], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->join_ev[q], cudaEventDisableTiming) != cudaSuccess) {
            delete ctx;
            return nullptr;
        }
    }
    if (cudaEventCreateWithFlags(&ctx->hc_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->hc_join, cudaEventDisableTiming) != cudaSuccess) {
        delete ctx;
        return nullptr;
    }
    ctx->stream = ctx->own_stream;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->cfg.device);
    {  // keep freed stream-ordered allocations in the pool (no release at synchronisations)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->cfg.device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    // the dimension gate's progress word; without it the dimensions simply join
    if (cudaHostAlloc(&ctx->h_gate, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->d_gate), ctx->h_gate, 0) != cudaSuccess ||
        cudaMallocHost(&ctx->h_tail, sizeof(int)) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->gate_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->h_gate) cudaFreeHost(ctx->h_gate);
        if (ctx->h_tail) cudaFreeHost(ctx->h_tail);
        if (ctx->gate_ev) cudaEventDestroy(ctx->gate_ev);
        ctx->h_gate = ctx->d_gate = ctx->h_tail = nullptr;
        ctx->gate_ev = nullptr;
    }
    if (cudaMallocHost(&ctx->h_err, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_counters, sizeof(long long) * CNT_NUM) != cudaSuccess ||
        cudaMallocHost(&ctx->h_info, sizeof(DimInfo)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_dimtot, sizeof(unsigned long long) * kNumDims) != cudaSuccess ||
        cudaMallocHost(&ctx->h_top, sizeof(unsigned long long)) != cudaSuccess) {
        delete ctx;
        return nullptr;
    }
    sspp_default_params(&ctx->params);
    return ctx;
}

void sspp_destroy(sspp_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->cfg.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_device(ctx->D);
    if (ctx->dropped) cudaFree(ctx->dropped);
    if (ctx->own_dims) cudaFree(ctx->own_dims);
    if (ctx->own_colptr) cudaFree(ctx->own_colptr);
    if (ctx->own_rows) cudaFree(ctx->own_rows);
    if (ctx->d_batch) cudaFree(ctx->d_batch);
    {
        void* q[] = {ctx->q_info, ctx->q_items, ctx->q_ctr, ctx->q_cplx, ctx->q_loff, ctx->q_lists, ctx->q_pool_c,
                     ctx->q_cstart, ctx->bvalues};
        for (void* p : q)
            if (p) cudaFree(p);
    }
    collapse_free(ctx->cs);
    build_free(ctx->bs);
    for (auto* t : ctx->hc.tup)
        if (t) cudaFree(t);
    if (ctx->hc.deg) cudaFree(ctx->hc.deg);
    if (ctx->hc.adj_off) cudaFree(ctx->hc.adj_off);
    if (ctx->hc.adj) cudaFree(ctx->hc.adj);
    if (ctx->hc.adj_src) cudaFree(ctx->hc.adj_src);
    if (ctx->hc.nmask) cudaFree(ctx->hc.nmask);
    if (ctx->hc.blk) cudaFree(ctx->hc.blk);
    if (ctx->hc.table) cudaFree(ctx->hc.table);
    ctx->prof.release();
    for (int q = 0; q < sspp_ctx::kSide; q++)
        if (ctx->side[q]) cudaStreamSynchronize(ctx->side[q]);
    for (auto ev : ctx->step_ev) cudaEventDestroy(ev);
    for (int q = 0; q < sspp_ctx::kSide; q++) {
        if (ctx->join_ev[q]) cudaEventDestroy(ctx->join_ev[q]);
        if (ctx->side[q]) cudaStreamDestroy(ctx->side[q]);
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    if (ctx->h_gate) cudaFreeHost(ctx->h_gate);
    if (ctx->h_tail) cudaFreeHost(ctx->h_tail);
    if (ctx->gate_ev) cudaEventDestroy(ctx->gate_ev);
    if (ctx->hc_fork) cudaEventDestroy(ctx->hc_fork);
    if (ctx->hc_join) cudaEventDestroy(ctx->hc_join);
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    if (ctx->h_info) cudaFreeHost(ctx->h_info);
    if (ctx->h_dimtot) cudaFreeHost(ctx->h_dimtot);
    if (ctx->h_top) cudaFreeHost(ctx->h_top);
    delete ctx;
}

const char* sspp_last_error(const sspp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t sspp_load_csc(sspp_ctx* ctx, int64_t ncols, const int32_t* dims, const int64_t* col_ptr, const int32_t* rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (ncols < 0 || (ncols > 0 && (!dims || !col_ptr)) || !col_ptr)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "null input array");
    // the rest of col_ptr (non-decreasing, column lengths) is checked on the device
    if (col_ptr[0] != 0 || col_ptr[ncols] < 0)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "col_ptr must start at 0 and be non-decreasing");
    const int64_t nnz = col_ptr[ncols];
    if (nnz > 0 && !rows) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null rows");
    int rc = load_common(ctx, ncols, nnz);
    if (rc) return rc;
    rc = ensure_own(ctx, ncols, nnz);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    const std::vector<Piece> pcs = {{dims, ctx->own_dims, sizeof(int32_t) * size_t(ncols)},
                                    {col_ptr, ctx->own_colptr, sizeof(int64_t) * size_t(ncols + 1)},
                                    {rows, ctx->own_rows, sizeof(int32_t) * size_t(nnz)}};
    CK(ctx->xfer.h2d(pcs, s));
    CK(cudaStreamSynchronize(s));
    ctx->D.in_dims = ctx->own_dims;
    ctx->D.in_colptr = ctx->own_colptr;
    ctx->D.in_rows = ctx->own_rows;
    ctx->loaded = true;
    return SSPP_OK;
}

int32_t sspp_load_csc_device(sspp_ctx* ctx, int64_t ncols, const int32_t* d_dims, const int64_t* d_col_ptr,
                             const int32_t* d_rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (ncols < 0 || !d_col_ptr || (ncols > 0 && !d_dims)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null input array");
    // col_ptr is checked on the device by the init pass; only its last entry is read here
    int64_t nnz = 0;
    CK(cudaMemcpyAsync(ctx->h_top, d_col_ptr + ncols, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::memcpy(&nnz, ctx->h_top, sizeof(int64_t));
    if (nnz < 0 || (nnz > 0 && !d_rows)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "col_ptr[ncols] out of range");
    int rc = load_common(ctx, ncols, nnz);
    if (rc) return rc;
    ctx->D.in_dims = const_cast<int32_t*>(d_dims);
    ctx->D.in_colptr = const_cast<int64_t*>(d_col_ptr);
    ctx->D.in_rows = const_cast<int32_t*>(d_rows);
    ctx->loaded = true;
    return SSPP_OK;
}

int32_t sspp_load_rips(sspp_ctx* ctx, int64_t npts, int32_t space_dim, const float* points, float radius,
                       int32_t maxdim) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (npts < 0 || (npts > 0 && !points) || space_dim < 1 || space_dim > 3)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad point array or space dimension");
    const auto t0 = std::chrono::steady_clock::now();
    ctx->loaded = false;  // the build reuses the buffers of an earlier build
    const float* dp = nullptr;
    if (npts > 0) {
        int rc = stage_floats(ctx, points, npts * space_dim, &dp);
        if (rc) return rc;
    }
    Built b;
    std::string msg;
    const int rc = build_rips(ctx->bs, dp, npts, space_dim, radius, maxdim, ctx->stream, &b, &msg);
    return finish_build(ctx, rc, b, msg, t0);
}

int32_t sspp_load_lowerstar(sspp_ctx* ctx, int64_t gx, int64_t gy, int64_t gz, const float* values,
                            int32_t maxdim) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (gx < 1 || gy < 1 || gz < 1 || !values || gx > INT32_MAX || gy > INT32_MAX || gz > INT32_MAX ||
        gx * gy > INT32_MAX || gx * gy * gz > INT32_MAX)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad grid size or null values");
    const auto t0 = std::chrono::steady_clock::now();
    ctx->loaded = false;
    const float* dv = nullptr;
    int rc = stage_floats(ctx, values, gx * gy * gz, &dv);
    if (rc) return rc;
    Built b;
    std::string msg;
    rc = build_lowerstar(ctx->bs, dv, gx, gy, gz, maxdim, ctx->stream, &b, &msg);
    return finish_build(ctx, rc, b, msg, t0);
}

int32_t sspp_input_size(sspp_ctx* ctx, int64_t* ncols, int64_t* nnz) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    if (!ctx->loaded) return set_err(ctx, SSPP_ERR_STATE, "nothing loaded");
    if (ncols) *ncols = ctx->D.n;
    if (nnz) *nnz = ctx->D.nnz;
    return SSPP_OK;
}

int32_t sspp_input_copy(sspp_ctx* ctx, int32_t* dims, int64_t* col_ptr, int32_t* rows, float* values) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->loaded) return set_err(ctx, SSPP_ERR_STATE, "nothing loaded");
    if (values && !ctx->built)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "filtration values exist for built complexes only");
    const Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    if (dims && D.n > 0) CK(cudaMemcpyAsync(dims, D.in_dims, sizeof(int32_t) * size_t(D.n), cudaMemcpyDeviceToHost, s));
    if (col_ptr)
        CK(cudaMemcpyAsync(col_ptr, D.in_colptr, sizeof(int64_t) * size_t(D.n + 1), cudaMemcpyDeviceToHost, s));
    if (rows && D.nnz > 0)
        CK(cudaMemcpyAsync(rows, D.in_rows, sizeof(int32_t) * size_t(D.nnz), cudaMemcpyDeviceToHost, s));
    if (values && D.n > 0)
        CK(cudaMemcpyAsync(values, ctx->built_batch ? ctx->bvalues : static_cast<float*>(ctx->bs.p[BuildScratch::VALUES]),
                           sizeof(float) * size_t(D.n), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return SSPP_OK;
}

int32_t sspp_load_built_batch(sspp_ctx* ctx, int32_t k, const sspp_build_spec* specs) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (k < 0 || (k > 0 && !specs)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null build specs");
    for (int32_t i = 0; i < k; i++) {
        const sspp_build_spec& b = specs[i];
        if (b.kind == SSPP_BUILD_RIPS) {
            if (b.size[0] < 0 || (b.size[0] > 0 && !b.data) || b.size[1] < 1 || b.size[1] > 3)
                return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad point array or space dimension");
        } else if (b.kind == SSPP_BUILD_LOWERSTAR) {
            const int64_t gx = b.size[0], gy = b.size[1], gz = b.size[2];
            if (gx < 1 || gy < 1 || gz < 1 || !b.data || gx > INT32_MAX || gy > INT32_MAX || gz > INT32_MAX ||
                gx * gy > INT32_MAX || gx * gy * gz > INT32_MAX)
                return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad grid size or null values");
        } else {
            return set_err(ctx, SSPP_ERR_BAD_INPUT, "unknown build kind");
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    ctx->loaded = false;
    cudaStream_t s = ctx->stream;
    std::vector<int64_t> starts(size_t(2) * (size_t(k) + 1), 0);  // column starts, then entry starts
    int64_t* cst = starts.data();
    int64_t* est = cst + k + 1;
    // each complex is built in the builder's buffers, then appended to the
    // context's input buffers (col_ptr entries and faces still local)
    for (int32_t i = 0; i < k; i++) {
        const sspp_build_spec& b = specs[i];
        const int64_t nin = b.kind == SSPP_BUILD_RIPS ? b.size[0] * b.size[1] : b.size[0] * b.size[1] * b.size[2];
        const float* din = nullptr;
        if (nin > 0) {
            int rc = stage_floats(ctx, b.data, nin, &din);
            if (rc) return rc;
        }
        Built out;
        std::string msg;
        const int rc = b.kind == SSPP_BUILD_RIPS
                           ? build_rips(ctx->bs, din, b.size[0], int(b.size[1]), b.radius, b.maxdim, s, &out, &msg)
                           : build_lowerstar(ctx->bs, din, b.size[0], b.size[1], b.size[2], b.maxdim, s, &out, &msg);
        if (rc) return set_err(ctx, rc == -1 ? SSPP_ERR_BAD_INPUT : SSPP_ERR_CUDA, msg);
        const int64_t n0 = cst[i], e0 = est[i];
        cst[i + 1] = n0 + out.ncols;
        est[i + 1] = e0 + out.nnz;
        if (cst[i + 1] > INT32_MAX - 8) return set_err(ctx, SSPP_ERR_CAPACITY, "more than 2^31 columns");
        CK(grow_own_cols(ctx, cst[i + 1] + 1, n0, s));
        CK(grow_keep(ctx->own_rows, ctx->cap_own_nnz, std::max<int64_t>(est[i + 1], 1), e0, s));
        CK(grow_keep(ctx->bvalues, ctx->cap_bvalues, std::max<int64_t>(cst[i + 1], 1), n0, s));
        if (out.ncols > 0) {
            CK(cudaMemcpyAsync(ctx->own_dims + n0, out.dims, sizeof(int32_t) * size_t(out.ncols),
                               cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(ctx->own_colptr + n0 + 1, out.col_ptr + 1, sizeof(int64_t) * size_t(out.ncols),
                               cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(ctx->bvalues + n0, out.values, sizeof(float) * size_t(out.ncols),
                               cudaMemcpyDeviceToDevice, s));
        }
        if (out.nnz > 0)
            CK(cudaMemcpyAsync(ctx->own_rows + e0, out.rows, sizeof(int32_t) * size_t(out.nnz),
                               cudaMemcpyDeviceToDevice, s));
    }
    const int64_t n = cst[k], nnz = est[k];
    CK(grow_own_cols(ctx, n + 1, n, s));
    if (!ctx->own_rows) CK(grow_keep(ctx->own_rows, ctx->cap_own_nnz, 1, 0, s));
    CK(cudaMemsetAsync(ctx->own_colptr, 0, sizeof(int64_t), s));
    CK(grow(ctx->d_batch, ctx->cap_d_batch, 2 * int64_t(starts.size()) + 1, s));
    CK(cudaMemcpyAsync(ctx->d_batch, starts.data(), sizeof(int64_t) * starts.size(), cudaMemcpyHostToDevice, s));
    int* d_bad = reinterpret_cast<int*>(ctx->d_batch + starts.size());
    CK(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    batch_rebase(n, nnz, k, ctx->d_batch, ctx->d_batch + k + 1, ctx->own_colptr, ctx->own_rows, d_bad, s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    int rc = load_common(ctx, n, nnz);
    if (rc) return rc;
    ctx->D.in_dims = ctx->own_dims;
    ctx->D.in_colptr = ctx->own_colptr;
    ctx->D.in_rows = ctx->own_rows;
    ctx->batch_start.assign(cst, cst + k + 1);
    ctx->loaded = true;
    ctx->built = true;
    ctx->built_batch = true;
    ctx->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SSPP_OK;
}

int64_t sspp_batch_values(sspp_ctx* ctx, int32_t i, float* out, int64_t cap) {
    if (!ctx) return -1;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->loaded || !ctx->built_batch || i < 0 || i + 1 >= int32_t(ctx->batch_start.size())) {
        set_err(ctx, SSPP_ERR_STATE, "no built batch loaded, or no complex of that index");
        return -1;
    }
    const int64_t b = ctx->batch_start[size_t(i)], e = ctx->batch_start[size_t(i) + 1];
    const int64_t m = std::min(cap, e - b);
    if (out && m > 0) {
        if (cudaMemcpyAsync(out, ctx->bvalues + b, sizeof(float) * size_t(m), cudaMemcpyDeviceToHost, ctx->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            set_err(ctx, SSPP_ERR_CUDA, "value copy failed");
            return -1;
        }
    }
    return e - b;
}

int32_t sspp_load_batch(sspp_ctx* ctx, int32_t k, const int64_t* ncols, const int32_t* const* dims,
                        const int64_t* const* col_ptr, const int32_t* const* rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (k < 0 || (k > 0 && (!ncols || !dims || !col_ptr || !rows)))
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "null batch arrays");
    std::vector<int64_t> starts(size_t(2) * (size_t(k) + 1), 0);  // column starts, then entry starts
    int64_t* cst = starts.data();
    int64_t* est = cst + k + 1;
    for (int32_t i = 0; i < k; i++) {
        if (ncols[i] < 0 || !col_ptr[i] || (ncols[i] > 0 && !dims[i]))
            return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad batch member");
        if (col_ptr[i][0] != 0 || col_ptr[i][ncols[i]] < 0)
            return set_err(ctx, SSPP_ERR_BAD_INPUT, "col_ptr must start at 0 and be non-decreasing");
        if (col_ptr[i][ncols[i]] > 0 && !rows[i]) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null rows");
        cst[i + 1] = cst[i] + ncols[i];
        est[i + 1] = est[i] + col_ptr[i][ncols[i]];
    }
    const int64_t n = cst[k], nnz = est[k];
    if (n > INT32_MAX - 8) return set_err(ctx, SSPP_ERR_CAPACITY, "more than 2^31 columns");
    int rc = load_common(ctx, n, nnz);
    if (rc) return rc;
    rc = ensure_own(ctx, n, nnz);
    if (rc) return rc;
    // starts (2 (k+1)), the bad-index flag, then the result slice starts (2 (k+1))
    CK(grow(ctx->d_batch, ctx->cap_d_batch, 2 * int64_t(starts.size()) + 1, ctx->stream));
    cudaStream_t s = ctx->stream;
    // the complexes side by side; indices are shifted on the device
    std::vector<Piece> pcs;
    pcs.reserve(size_t(3) * size_t(k) + 1);
    for (int32_t i = 0; i < k; i++)
        pcs.push_back({dims[i], ctx->own_dims + cst[i], sizeof(int32_t) * size_t(ncols[i]), 0});
    for (int32_t i = 0; i < k; i++)
        pcs.push_back({col_ptr[i] + 1, ctx->own_colptr + cst[i] + 1, sizeof(int64_t) * size_t(ncols[i]), 1});
    for (int32_t i = 0; i < k; i++)
        pcs.push_back({rows[i], ctx->own_rows + est[i], sizeof(int32_t) * size_t(est[i + 1] - est[i]), 2});
    pcs.push_back({starts.data(), ctx->d_batch, sizeof(int64_t) * starts.size(), 3});
    int* d_bad = reinterpret_cast<int*>(ctx->d_batch + starts.size());
    CK(cudaMemsetAsync(ctx->own_colptr, 0, sizeof(int64_t), s));
    CK(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    CK(ctx->xfer.h2d(pcs, s));
    batch_rebase(n, nnz, k, ctx->d_batch, ctx->d_batch + k + 1, ctx->own_colptr, ctx->own_rows, d_bad, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_err, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*ctx->h_err) {
        ctx->loaded = false;
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "a face index lies outside its own complex");
    }
    ctx->D.in_dims = ctx->own_dims;
    ctx->D.in_colptr = ctx->own_colptr;
    ctx->D.in_rows = ctx->own_rows;
    ctx->loaded = true;
    ctx->batch_start.assign(cst, cst + k + 1);
    return SSPP_OK;
}

int32_t sspp_load_batch_device(sspp_ctx* ctx, int32_t k, const int64_t* ncols, const int32_t* d_dims,
                               const int64_t* d_col_ptr, const int32_t* d_rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    if (k < 0 || (k > 0 && !ncols)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null batch sizes");
    std::vector<int64_t> starts(size_t(k) + 1, 0);
    for (int32_t i = 0; i < k; i++) {
        if (ncols[i] < 0) return set_err(ctx, SSPP_ERR_BAD_INPUT, "negative batch member size");
        starts[size_t(i) + 1] = starts[size_t(i)] + ncols[i];
    }
    int rc = sspp_load_csc_device(ctx, starts[size_t(k)], d_dims, d_col_ptr, d_rows);
    if (rc) return rc;
    CK(grow(ctx->d_batch, ctx->cap_d_batch, 4 * (int64_t(k) + 1) + 1, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_batch, starts.data(), sizeof(int64_t) * starts.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->batch_start = starts;
    return SSPP_OK;
}

// pairs of complex i, in its own indices (the sorted global pairs are copied once)
static int batch_slice(sspp_ctx* ctx, int32_t i, int64_t& b, int64_t& e) {
    if (!ctx->computed || ctx->batch_start.empty() || i < 0 || i + 1 >= int32_t(ctx->batch_start.size()))
        return SSPP_ERR_STATE;
    if (!ctx->host_pairs_valid) {
        const int64_t k = ctx->hcounters[CNT_NPAIRS];
        ctx->host_pairs.resize(size_t(2 * k));
        if (k > 0 && ctx->xfer.d2h({{ctx->D.pairs, ctx->host_pairs.data(), sizeof(int64_t) * 2 * size_t(k)}},
                                   ctx->stream) != cudaSuccess)
            return SSPP_ERR_CUDA;
        ctx->host_pairs_valid = true;
    }
    const int64_t npairs = int64_t(ctx->host_pairs.size() / 2);
    const int64_t lo = ctx->batch_start[size_t(i)], hi = ctx->batch_start[size_t(i) + 1];
    auto first_at_least = [&](int64_t x) {  // first pair whose birth >= x
        int64_t l = 0, h = npairs;
        while (l < h) {
            int64_t m = (l + h) / 2;
            if (ctx->host_pairs[size_t(2 * m)] < x) l = m + 1;
            else h = m;
        }
        return l;
    };
    b = first_at_least(lo);
    e = first_at_least(hi);
    return SSPP_OK;
}

int64_t sspp_batch_num_pairs(sspp_ctx* ctx, int32_t i) {
    if (!ctx) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t b, e;
    if (batch_slice(ctx, i, b, e)) return -1;
    return e - b;
}

int64_t sspp_batch_pairs(sspp_ctx* ctx, int32_t i, int64_t* out, int64_t cap) {
    if (!ctx || cap < 0 || (!out && cap > 0)) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t b, e;
    if (batch_slice(ctx, i, b, e)) return -1;
    const int64_t off = ctx->batch_start[size_t(i)];
    const int64_t n = std::min(cap, e - b);
    for (int64_t t = 0; t < n; t++) {
        out[2 * t] = ctx->host_pairs[size_t(2 * (b + t))] - off;
        out[2 * t + 1] = ctx->host_pairs[size_t(2 * (b + t) + 1)] - off;
    }
    return n;
}

// essentials of complex i (the ascending global list is copied once)
static int batch_ess_slice(sspp_ctx* ctx, int32_t i, int64_t& b, int64_t& e) {
    if (!ctx->computed || ctx->batch_start.empty() || i < 0 || i + 1 >= int32_t(ctx->batch_start.size()))
        return SSPP_ERR_STATE;
    if (!ctx->host_ess_valid) {
        const int64_t k = ctx->hcounters[CNT_NESS];
        ctx->host_ess.resize(size_t(k));
        if (k > 0 && ctx->xfer.d2h({{ctx->D.ess, ctx->host_ess.data(), sizeof(int64_t) * size_t(k)}}, ctx->stream) !=
                         cudaSuccess)
            return SSPP_ERR_CUDA;
        ctx->host_ess_valid = true;
    }
    const auto& v = ctx->host_ess;
    b = std::lower_bound(v.begin(), v.end(), ctx->batch_start[size_t(i)]) - v.begin();
    e = std::lower_bound(v.begin(), v.end(), ctx->batch_start[size_t(i) + 1]) - v.begin();
    return SSPP_OK;
}

int64_t sspp_batch_num_essential(sspp_ctx* ctx, int32_t i) {
    if (!ctx) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t b, e;
    if (batch_ess_slice(ctx, i, b, e)) return -1;
    return e - b;
}

int64_t sspp_batch_essentials(sspp_ctx* ctx, int32_t i, int64_t* out, int64_t cap) {
    if (!ctx || cap < 0 || (!out && cap > 0)) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t b, e;
    if (batch_ess_slice(ctx, i, b, e)) return -1;
    const int64_t off = ctx->batch_start[size_t(i)];
    const int64_t n = std::min(cap, e - b);
    for (int64_t t = 0; t < n; t++) out[t] = ctx->host_ess[size_t(b + t)] - off;
    return n;
}

// Bulk results of a batch: per-complex counts, then one staged copy of every
// complex's pairs and essentials (indices made local on the device).
int32_t sspp_batch_counts(sspp_ctx* ctx, int64_t* npairs, int64_t* ness) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->computed || ctx->batch_start.empty()) return set_err(ctx, SSPP_ERR_STATE, "no reduced batch");
    const int32_t k = int32_t(ctx->batch_start.size()) - 1;
    const int64_t np = ctx->hcounters[CNT_NPAIRS], ne = ctx->hcounters[CNT_NESS];
    int64_t* d_cstart = ctx->d_batch;
    int64_t* d_ps = ctx->d_batch + 2 * (int64_t(k) + 1) + 1;
    int64_t* d_es = d_ps + k + 1;
    cudaStream_t s = ctx->stream;
    batch_bounds(k, d_cstart, np, ctx->D.pairs, ne, ctx->D.ess, d_ps, d_es, s);
    ctx->batch_bounds.resize(2 * (size_t(k) + 1));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->batch_bounds.data(), d_ps, sizeof(int64_t) * 2 * (size_t(k) + 1), cudaMemcpyDeviceToHost,
                       s));
    CK(cudaStreamSynchronize(s));
    const int64_t* ps = ctx->batch_bounds.data();
    const int64_t* es = ps + k + 1;
    for (int32_t i = 0; i < k; i++) {
        if (npairs) npairs[i] = (i + 1 < k ? ps[i + 1] : np) - ps[i];
        if (ness) ness[i] = (i + 1 < k ? es[i + 1] : ne) - es[i];
    }
    return SSPP_OK;
}

int32_t sspp_batch_copy(sspp_ctx* ctx, int64_t* const* pairs_out, int64_t* const* ess_out) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    const int32_t k = int32_t(ctx->batch_start.size()) - 1;
    if (!ctx->computed || k < 0 || ctx->batch_bounds.size() != 2 * (size_t(k) + 1))
        return set_err(ctx, SSPP_ERR_STATE, "call sspp_batch_counts first");
    const int64_t np = ctx->hcounters[CNT_NPAIRS], ne = ctx->hcounters[CNT_NESS];
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    // local copies live in buffers the reduction no longer needs: 2 np <= n, ne <= n
    int64_t* lp = D.death_of;
    int64_t* le = D.scratch64;
    batch_localize(np, ne, k, ctx->d_batch, D.pairs, D.ess, lp, le, s);
    CK(cudaGetLastError());
    const int64_t* ps = ctx->batch_bounds.data();
    const int64_t* es = ps + k + 1;
    std::vector<Piece> pcs;
    pcs.reserve(2 * size_t(k));
    for (int32_t i = 0; i < k; i++) {
        const int64_t a = ps[i], b = i + 1 < k ? ps[i + 1] : np;
        if (b > a && pairs_out && pairs_out[i])
            pcs.push_back({lp + 2 * a, pairs_out[i], sizeof(int64_t) * 2 * size_t(b - a), -1});
    }
    for (int32_t i = 0; i < k; i++) {
        const int64_t a = es[i], b = i + 1 < k ? es[i + 1] : ne;
        if (b > a && ess_out && ess_out[i]) pcs.push_back({le + a, ess_out[i], sizeof(int64_t) * size_t(b - a), -1});
    }
    CK(ctx->xfer.d2h(pcs, s));
    return SSPP_OK;
}

int32_t sspp_load_phat(sspp_ctx* ctx, const char* path, int32_t fmt) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    if (!path || (fmt != SSPP_ASCII && fmt != SSPP_BINARY)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad path or format");
    PhatMatrix m;
    std::string e;
    if (!read_phat(path, fmt, m, e)) return set_err(ctx, SSPP_ERR_IO, e);
    return sspp_load_csc(ctx, int64_t(m.dims.size()), m.dims.data(), m.col_ptr.data(), m.rows.data());
}

int32_t sspp_init(sspp_ctx* ctx, const sspp_params* p, void* stream) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->loaded) return set_err(ctx, SSPP_ERR_STATE, "no matrix loaded");
    int rc = check_params(ctx, p);
    if (rc) return rc;
    ctx->params = *p;
    ctx->user_params = *p;
    ctx->tune_cand = -1;
    ctx->tune_locked = false;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return run_init(ctx);
}

int32_t sspp_compute(sspp_ctx* ctx, void* stream) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->inited) return set_err(ctx, SSPP_ERR_STATE, "sspp_init has not completed");
    if (stream) ctx->stream = static_cast<cudaStream_t>(stream);
    for (int attempt = 0; attempt < 6; attempt++) {
        int rc = run_compute(ctx);
        if (rc == SSPP_OK && ctx->tune_cand >= 0) {
            const sspp_params& u = ctx->user_params;
            const double base = double(ctx->D.nnz + (kHdr + 3) * ctx->D.n + 4);
            tune_record(ctx->D.n, ctx->tune_shape, u.model, u.dualize, tune_allows_dual(u), ctx->tune_cand,
                        ctx->init_ms + ctx->compute_ms, double(ctx->arena_used) / base);
        }
        if (rc != SSPP_ERR_CAPACITY || !ctx->err.empty()) return rc;
        ctx->tune_locked = true;  // the repeat keeps this run's choice
        // arena or heavy pool exhausted: grow both and redo the whole reduction from the input
        ctx->arena_request = std::max<int64_t>(ctx->D.arena_cap * 2, arena_need(ctx));
        ctx->pool_request = std::max<int64_t>(ctx->D.pool_cap * 2, 1 << 16);
        rc = run_init(ctx);
        if (rc) return rc;
    }
    return set_err(ctx, SSPP_ERR_CAPACITY, "device arena exhausted");
}

int32_t sspp_reduce(sspp_ctx* ctx, const sspp_params* p, void* stream) {
    int rc = sspp_init(ctx, p, stream);
    if (rc) return rc;
    return sspp_compute(ctx, stream);
}

int64_t sspp_num_pairs(sspp_ctx* ctx) {
    if (!ctx || !ctx->computed) return -1;
    return ctx->hcounters[CNT_NPAIRS];
}

int64_t sspp_pairs(sspp_ctx* ctx, int64_t* out, int64_t cap) {
    if (!ctx || !ctx->computed || cap < 0 || (!out && cap > 0)) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t n = std::min<int64_t>(cap, ctx->hcounters[CNT_NPAIRS]);
    if (n > 0 && ctx->xfer.d2h({{ctx->D.pairs, out, sizeof(int64_t) * 2 * size_t(n)}}, ctx->stream) != cudaSuccess) {
        set_err(ctx, SSPP_ERR_CUDA, "pairs copy failed");
        return -1;
    }
    return n;
}

int64_t sspp_num_essential(sspp_ctx* ctx) {
    if (!ctx || !ctx->computed) return -1;
    return ctx->hcounters[CNT_NESS];
}

int64_t sspp_essentials(sspp_ctx* ctx, int64_t* out, int64_t cap) {
    if (!ctx || !ctx->computed || cap < 0 || (!out && cap > 0)) return -1;
    cudaSetDevice(ctx->cfg.device);
    int64_t n = std::min<int64_t>(cap, ctx->hcounters[CNT_NESS]);
    if (n > 0 && cudaMemcpy(out, ctx->D.ess, sizeof(int64_t) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err(ctx, SSPP_ERR_CUDA, "essentials copy failed");
        return -1;
    }
    return n;
}

int32_t sspp_export_preprocessed(sspp_ctx* ctx, const sspp_params* p, const char* path, int32_t fmt) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (!ctx->loaded) return set_err(ctx, SSPP_ERR_STATE, "no matrix loaded");
    if (!path || (fmt != SSPP_ASCII && fmt != SSPP_BINARY)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "bad path or format");
    int rc = check_params(ctx, p);
    if (rc) return rc;
    ctx->params = *p;
    ctx->inited = ctx->computed = false;
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    const int64_t n = D.n, nnz = D.nnz;
    std::vector<int32_t> dims(size_t(std::max<int64_t>(n, 1)));
    std::vector<int64_t> cp(size_t(n) + 1, 0);
    std::vector<int32_t> rows(size_t(std::max<int64_t>(nnz, 1)));
    if (n > 0) {
        CK(cudaMemcpyAsync(dims.data(), D.in_dims, 4 * size_t(n), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(cp.data(), D.in_colptr, 8 * (size_t(n) + 1), cudaMemcpyDeviceToHost, s));
    }
    if (nnz > 0) CK(cudaMemcpyAsync(rows.data(), D.in_rows, 4 * size_t(nnz), cudaMemcpyDeviceToHost, s));
    CK(cudaMemsetAsync(D.err, 0, sizeof(int), s));
    CK(cudaMemsetAsync(D.counters, 0, sizeof(long long) * CNT_NUM, s));
    CK(cudaStreamSynchronize(s));
    std::vector<uint8_t> drop(size_t(std::max<int64_t>(n, 1)), 0);
    if (n > 0 && (p->model & 3)) {
        rc = ensure_arena(ctx, arena_need(ctx));
        if (rc) return rc;
        validate(D, s);
        CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (*ctx->h_err) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dimension out of range 0..7 or malformed col_ptr");
        reorder(D, false, s);
        CK(cudaMemcpyAsync(D.arena_top, D.blk + reorder_total_slot(D), sizeof(unsigned long long),
                           cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (*ctx->h_err) return set_err(ctx, SSPP_ERR_BAD_INPUT, "malformed boundary matrix");
        if (p->model & 2) {
            rc = run_collapse(ctx);
            if (rc) return rc;
        }
        CK(cudaMemsetAsync(D.cleared, 0, size_t(n), s));
        if ((p->model & 1) && p->max_iteration > 0) {
            rc = run_highclear(ctx, ctx->stream);
            if (rc) return rc;
        }
        std::vector<int32_t> perm(static_cast<size_t>(n));
        std::vector<uint8_t> cl(static_cast<size_t>(n)), dr(static_cast<size_t>(n), 0);
        CK(cudaMemcpyAsync(perm.data(), D.perm, 4 * size_t(n), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(cl.data(), D.cleared, size_t(n), cudaMemcpyDeviceToHost, s));
        if (p->model & 2) CK(cudaMemcpyAsync(dr.data(), ctx->dropped, size_t(n), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(ctx->h_counters, D.counters, sizeof(long long) * CNT_NUM, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        CK(cudaGetLastError());
        std::memcpy(ctx->hcounters, ctx->h_counters, sizeof(ctx->hcounters));
        for (int64_t i = 0; i < n; i++)
            if (cl[size_t(i)] || dr[size_t(i)]) drop[size_t(perm[size_t(i)])] = 1;
    }
    // cleared and dropped columns become dimension-only lines (include/specseq.h:1115-1123)
    std::vector<int64_t> ocp(size_t(n) + 1, 0);
    std::vector<int32_t> orows;
    orows.reserve(size_t(std::max<int64_t>(nnz, 1)));
    for (int64_t j = 0; j < n; j++) {
        if (!drop[size_t(j)]) orows.insert(orows.end(), rows.begin() + cp[size_t(j)], rows.begin() + cp[size_t(j) + 1]);
        ocp[size_t(j) + 1] = int64_t(orows.size());
    }
    std::string e;
    if (!write_phat(path, fmt, n, dims.data(), ocp.data(), orows.data(), e)) return set_err(ctx, SSPP_ERR_IO, e);
    return SSPP_OK;
}

int32_t sspp_write_pairs(sspp_ctx* ctx, const char* path, int32_t fmt) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    if (!ctx->computed) return set_err(ctx, SSPP_ERR_STATE, "no pairs computed");
    int64_t n = ctx->hcounters[CNT_NPAIRS];
    std::vector<int64_t> bd(size_t(2 * n));
    if (sspp_pairs(ctx, bd.data(), n) != n) return SSPP_ERR_CUDA;
    std::string e;
    if (!write_pairs(path, fmt, bd.data(), n, e)) return set_err(ctx, SSPP_ERR_IO, e);
    return SSPP_OK;
}

int32_t sspp_get_params(const sspp_ctx* ctx, sspp_params* out) {
    if (!ctx || !out) return SSPP_ERR_BAD_INPUT;
    *out = ctx->params;
    return SSPP_OK;
}

int64_t sspp_representative(sspp_ctx* ctx, int64_t death, int64_t* out, int64_t cap) {
    if (!ctx) return -1;
    cudaSetDevice(ctx->cfg.device);
    auto fail = [&](int code, const char* msg) -> int64_t {
        set_err(ctx, code, msg);
        return -1;
    };
    if (!ctx->computed) return fail(SSPP_ERR_STATE, "no completed reduction");
    if (!ctx->params.representatives) return fail(SSPP_ERR_STATE, "the reduction ran without representatives = 1");
    if (!ctx->batch_start.empty()) return fail(SSPP_ERR_STATE, "representatives are not kept for batches");
    const Device& D = ctx->D;
    if (death < 0 || death >= D.n) return fail(SSPP_ERR_BAD_INPUT, "death index out of range");
    if (cap > 0 && !out) return fail(SSPP_ERR_BAD_INPUT, "null output");
    cudaStream_t s = ctx->stream;
    // the death's reordered column, its descriptor, and the owner of its lowest row
    int32_t c = 0;
    uint64_t d = 0;
    if (cudaMemcpyAsync(&c, D.newidx + death, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess || c < 0 || c >= D.n ||
        cudaMemcpyAsync(&d, D.desc + c, sizeof(uint64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(SSPP_ERR_CUDA, "reading the death column failed");
    const uint32_t len = desc_len(d);
    if (len == 0) return fail(SSPP_ERR_BAD_INPUT, "not a death: the column reduced to zero");
    std::vector<int32_t> rows(len);
    uint64_t e = 0;
    if (cudaMemcpyAsync(rows.data(), D.arena + desc_off(d) + kHdr, sizeof(int32_t) * len, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess || rows.back() < 0 || rows.back() >= D.n ||
        cudaMemcpyAsync(&e, D.pivot + rows.back(), sizeof(uint64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(SSPP_ERR_CUDA, "reading the reduced column failed");
    if (e == kNoOwner || pv_col(e) != c) return fail(SSPP_ERR_BAD_INPUT, "not a death: the column owns no row");
    if (!ctx->host_perm_valid) {
        ctx->host_perm.resize(size_t(D.n));
        if (cudaMemcpyAsync(ctx->host_perm.data(), D.perm, sizeof(int32_t) * size_t(D.n), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail(SSPP_ERR_CUDA, "reading the index map failed");
        ctx->host_perm_valid = true;
    }
    std::vector<int64_t> cyc(len);
    for (uint32_t k = 0; k < len; k++) {
        if (rows[k] < 0 || rows[k] >= D.n) return fail(SSPP_ERR_BAD_INPUT, "row index out of range");
        cyc[k] = ctx->host_perm[size_t(rows[k])];
    }
    std::sort(cyc.begin(), cyc.end());
    for (int64_t k = 0; k < std::min<int64_t>(cap, len); k++) out[k] = cyc[size_t(k)];
    return int64_t(len);
}

int32_t sspp_get_stats(const sspp_ctx* ctx, sspp_stats* o) {
    if (!ctx || !o) return SSPP_ERR_BAD_INPUT;
    std::memset(o, 0, sizeof(*o));
    const long long* c = ctx->hcounters;
    o->ncols = ctx->D.n;
    o->nnz = ctx->D.nnz;
    o->active_after_init = c[CNT_ACTIVE];
    o->apparent_pairs = c[CNT_APPARENT];
    o->cleared_init = c[CNT_CLEARED];
    o->highclear_cleared = c[CNT_HIGHCLEAR];
    o->collapse_dropped = c[CNT_DROPPED];
    o->arena_ints_used = ctx->arena_used;
    o->tuned_candidate = ctx->tune_cand;
    o->heavy_additions = c[CNT_HEAVY_ADDS];
    o->additions = c[CNT_ADDITIONS];
    o->add_ints = c[CNT_ADD_INTS];
    o->published_ints = c[CNT_PUBLISHED];
    o->displaced = c[CNT_DISPLACED];
    o->ss_steps = ctx->ss_steps;
    o->npairs = ctx->computed ? c[CNT_NPAIRS] : 0;
    o->nessential = ctx->computed ? c[CNT_NESS] : 0;
    o->init_ms = ctx->init_ms;
    o->compute_ms = ctx->compute_ms;
    o->launches = ctx->launches;
    o->init_gpu_ms = ctx->ph_ms[PH_INIT];
    o->light_gpu_ms = ctx->ph_ms[PH_LIGHT];
    o->heavy_gpu_ms = ctx->ph_ms[PH_HEAVY];
    o->pairs_gpu_ms = ctx->ph_ms[PH_PAIRS];
    o->light_launches = ctx->light_launches;
    o->heavy_launches = ctx->heavy_launches;
    o->build_ms = ctx->build_ms;
    o->heavy_fast_inline = c[CNT_FAST_INLINE];
    o->heavy_fast_slot = c[CNT_FAST_SLOT];
    return SSPP_OK;
}

}  // extern "C"
