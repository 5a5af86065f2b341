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
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "sspp_internal.h"
#include "sspp_io.h"
#include "sspp_launch.h"

using namespace sspp;

struct sspp_ctx {
    sspp_config cfg{};
    std::string err;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    Device D;
    sspp_params params{};
    bool loaded = false, inited = false, computed = false;
    DimInfo hinfo{};
    long long hcounters[CNT_NUM] = {};
    int num_sms = 0;
    int blocks_per_sm = 0;
    int configured_cap = -1;
    int64_t arena_request = 0;     // ints requested for the arena (grows on CAPACITY)
    double init_ms = 0, compute_ms = 0;
    int64_t ss_steps = 0;
    int* h_err = nullptr;          // pinned
    long long* h_counters = nullptr;
    DimInfo* h_info = nullptr;
    unsigned long long* h_top = nullptr;
    uint8_t* dropped = nullptr;    // primal reordered numbering (model bit 2)
    int64_t cap_dropped = 0;
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

template <typename T>
cudaError_t grow(T*& p, int64_t& cap, int64_t want) {
    if (want <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, size_t(std::max<int64_t>(want, 1)) * sizeof(T));
    if (e == cudaSuccess) cap = want;
    return e;
}

void free_device(Device& D) {
    void* ptrs[] = {D.in_dims, D.in_colptr, D.in_rows, D.dim, D.perm, D.newidx, D.scratch64, D.arena, D.arena_top,
                    D.desc, D.low, D.pivot, D.state, D.cleared, D.negative, D.leftmost, D.active, D.blk, D.dimcnt,
                    D.diminfo, D.err, D.counters, D.step_ctr, D.death_of, D.pairs, D.ess};
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
            if (p) { cudaFree(p); p = nullptr; }
            return grow<T>(p, cap, c * mult + 1);
        };
        CK(g(D.in_dims, 1));
        CK(g(D.in_colptr, 1));
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
        CK(g(D.death_of, 1));
        CK(g(D.pairs, 2));
        CK(g(D.ess, 1));
        D.cap_n = c;
        int64_t nb = (c + 4095) / 4096 + 2;
        CK(grow(D.blk, D.cap_blk, nb));
        int64_t nbp = (c + 255) / 256 + 1;
        CK(grow(D.dimcnt, D.cap_dimcnt, nbp * kNumDims));
    }
    if (nnz > D.cap_nnz) {
        if (D.in_rows) cudaFree(D.in_rows);
        D.in_rows = nullptr;
        int64_t cap = 0;
        CK(grow(D.in_rows, cap, nnz));
        D.cap_nnz = nnz;
    }
    if (!D.diminfo) {
        CK(cudaMalloc(&D.diminfo, sizeof(DimInfo)));
        CK(cudaMalloc(&D.err, sizeof(int)));
        CK(cudaMalloc(&D.counters, sizeof(long long) * CNT_NUM));
        CK(cudaMalloc(&D.arena_top, sizeof(unsigned long long)));
    }
    return SSPP_OK;
}

int ensure_arena(sspp_ctx* ctx, int64_t ints) {
    Device& D = ctx->D;
    if (ints <= D.arena_cap) return SSPP_OK;
    if (D.arena) cudaFree(D.arena);
    D.arena = nullptr;
    D.arena_cap = 0;
    CK(cudaMalloc(&D.arena, size_t(ints) * sizeof(int32_t)));
    D.arena_cap = ints;
    return SSPP_OK;
}

int64_t arena_need(const sspp_ctx* ctx) {
    const int64_t base = ctx->D.nnz + 3 * ctx->D.n + 4;
    int64_t want = base + std::max<int64_t>(2 * base, int64_t(16) << 20);
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
    if (p->dualize != 0 && p->dualize != 1) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dualize must be 0 or 1");
    if (p->model < 0 || p->model > 3) return set_err(ctx, SSPP_ERR_BAD_INPUT, "model must be 0..3");
    if (p->max_iteration < 0) return set_err(ctx, SSPP_ERR_BAD_INPUT, "max_iteration must be >= 0");
    if (p->ss_block_size < 1) return set_err(ctx, SSPP_ERR_BAD_INPUT, "ss_block_size must be >= 1");
    if (!(p->growth >= 1.0f) || !std::isfinite(p->growth))
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "block_size_growth_rate must be >= 1");
    if (p->queue_size < 1) return set_err(ctx, SSPP_ERR_BAD_INPUT, "queue_size must be >= 1");
    if (p->level1_capacity < 0 || p->level2_capacity < 0)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "level capacities must be >= 0");
    if (p->dualize) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dualize is not available in this build");
    if (p->model & 3) return set_err(ctx, SSPP_ERR_BAD_INPUT, "model bits are not available in this build");
    return SSPP_OK;
}

int level1_cap(const sspp_params& p) {
    int c = std::max(64, p.level1_capacity);
    c = std::min(c, 4096);
    return (c + 31) & ~31;
}

int run_init(sspp_ctx* ctx) {
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    CK(cudaMemsetAsync(D.err, 0, sizeof(int), s));
    CK(cudaMemsetAsync(D.counters, 0, sizeof(long long) * CNT_NUM, s));
    int rc = ensure_arena(ctx, arena_need(ctx));
    if (rc) return rc;
    validate(D, s);
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*ctx->h_err) return set_err(ctx, SSPP_ERR_BAD_INPUT, "dimension out of range 0..7 or malformed col_ptr");
    reorder(D, s);
    CK(cudaMemcpyAsync(D.arena_top, D.blk + reorder_total_slot(D), sizeof(unsigned long long),
                       cudaMemcpyDeviceToDevice, s));
    init_passes(D, s);
    init_compress(D, nullptr, s);
    active_list(D, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_info, D.diminfo, sizeof(DimInfo), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_counters, D.counters, sizeof(long long) * CNT_NUM, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->hinfo = *ctx->h_info;
    std::memcpy(ctx->hcounters, ctx->h_counters, sizeof(ctx->hcounters));
    ctx->init_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (*ctx->h_err & ERRB_BAD_INPUT)
        return set_err(ctx, SSPP_ERR_BAD_INPUT,
                       "malformed boundary matrix (a face index out of range, unsorted, duplicated, or of the "
                       "wrong dimension)");
    if (*ctx->h_err) return set_err(ctx, SSPP_ERR_CAPACITY, "init pass overflow");
    ctx->inited = true;
    ctx->computed = false;
    return SSPP_OK;
}

int run_compute(sspp_ctx* ctx) {
    ctx->err.clear();
    Device& D = ctx->D;
    cudaStream_t s = ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    const sspp_params& P = ctx->params;
    const int cap = level1_cap(P);
    if (cap != ctx->configured_cap) {
        CK(reduce_configure(cap, &ctx->blocks_per_sm));
        ctx->configured_cap = cap;
        if (ctx->blocks_per_sm < 1) return set_err(ctx, SSPP_ERR_CAPACITY, "level1 capacity too large for shared memory");
    }
    // schedule (dimensions high to low)
    std::vector<Step> steps;
    std::vector<int> step_dim;
    const DimInfo& I = ctx->hinfo;
    for (int d = kMaxDim; d >= 1; d--) {
        size_t before = steps.size();
        ss_schedule(P, I.act_begin[d], I.act_end[d], I.min_row[d] == INT_MAX ? 0 : I.min_row[d], I.max_row[d], steps);
        for (size_t k = before; k < steps.size(); k++) step_dim.push_back(d);
    }
    if (int64_t(steps.size()) > D.cap_steps) {
        if (D.step_ctr) cudaFree(D.step_ctr);
        D.step_ctr = nullptr;
        D.cap_steps = 0;
        CK(grow(D.step_ctr, D.cap_steps, int64_t(steps.size()) + 64));
    }
    if (!steps.empty()) CK(cudaMemsetAsync(D.step_ctr, 0, sizeof(int) * steps.size(), s));
    const int max_blocks = std::max(1, ctx->num_sms * ctx->blocks_per_sm);
    const int q_blocks = std::max(1, (P.queue_size + 3) / 4);
    for (size_t k = 0; k < steps.size(); k++) {
        const Step& st = steps[k];
        int64_t chunks = (int64_t(st.end - st.beg) + 31) / 32;
        int grid = int(std::min<int64_t>(std::min<int64_t>((chunks + 3) / 4, max_blocks), q_blocks));
        grid = std::max(grid, 1);
        reduce_launch(D, D.active, st.beg, st.end, st.minrow, cap, D.step_ctr + k, grid, s);
    }
    ctx->ss_steps = int64_t(steps.size());
    extract_pairs(D, 0, nullptr, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_err, D.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ctx->h_counters, D.counters, sizeof(long long) * CNT_NUM, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::memcpy(ctx->hcounters, ctx->h_counters, sizeof(ctx->hcounters));
    ctx->compute_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const int e = *ctx->h_err;
    if (e & ERRB_CAPACITY) return SSPP_ERR_CAPACITY;
    if (e & ERRB_LEN) return set_err(ctx, SSPP_ERR_CAPACITY, "a column exceeded 2^24 entries");
    if (e & ERRB_TIMEOUT) return set_err(ctx, SSPP_ERR_TIMEOUT, "per-column merge limit reached");
    if (e) return set_err(ctx, SSPP_ERR_BAD_INPUT, "device error word set");
    ctx->computed = true;
    return SSPP_OK;
}

int load_common(sspp_ctx* ctx, int64_t n, int64_t nnz) {
    ctx->loaded = ctx->inited = ctx->computed = false;
    int rc = ensure_columns(ctx, n, nnz);
    if (rc) return rc;
    ctx->D.n = n;
    ctx->D.nnz = nnz;
    ctx->arena_request = 0;
    return SSPP_OK;
}

bool validate_colptr(const int64_t* cp, int64_t n) {
    if (cp[0] != 0) return false;
    for (int64_t j = 0; j < n; j++)
        if (cp[j + 1] < cp[j] || cp[j + 1] - cp[j] > kMaxColLen) return false;
    return true;
}

}  // namespace

extern "C" {

void sspp_default_params(sspp_params* p) {
    if (!p) return;
    p->dualize = 0;
    p->model = 0;
    p->max_iteration = 0;
    p->ss_block_size = 102400;
    p->growth = 1.05f;
    p->queue_size = 65536;
    p->level1_capacity = 1000;
    p->level2_capacity = 8000;
    p->autotune = 0;
}

sspp_ctx* sspp_create(const sspp_config* cfg) {
    auto* ctx = new (std::nothrow) sspp_ctx;
    if (!ctx) return nullptr;
    if (cfg) ctx->cfg = *cfg;
    if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) { delete ctx; return nullptr; }
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return nullptr; }
    ctx->stream = ctx->own_stream;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->cfg.device);
    if (cudaMallocHost(&ctx->h_err, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_counters, sizeof(long long) * CNT_NUM) != cudaSuccess ||
        cudaMallocHost(&ctx->h_info, sizeof(DimInfo)) != cudaSuccess ||
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
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    if (ctx->h_info) cudaFreeHost(ctx->h_info);
    if (ctx->h_top) cudaFreeHost(ctx->h_top);
    delete ctx;
}

const char* sspp_last_error(const sspp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t sspp_load_csc(sspp_ctx* ctx, int64_t ncols, const int32_t* dims, const int64_t* col_ptr, const int32_t* rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (ncols < 0 || (ncols > 0 && (!dims || !col_ptr)) || !col_ptr)
        return set_err(ctx, SSPP_ERR_BAD_INPUT, "null input array");
    if (!validate_colptr(col_ptr, ncols)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "col_ptr must start at 0 and be non-decreasing");
    const int64_t nnz = col_ptr[ncols];
    if (nnz > 0 && !rows) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null rows");
    int rc = load_common(ctx, ncols, nnz);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    if (ncols) CK(cudaMemcpyAsync(ctx->D.in_dims, dims, sizeof(int32_t) * ncols, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->D.in_colptr, col_ptr, sizeof(int64_t) * (ncols + 1), cudaMemcpyHostToDevice, s));
    if (nnz) CK(cudaMemcpyAsync(ctx->D.in_rows, rows, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    ctx->loaded = true;
    return SSPP_OK;
}

int32_t sspp_load_csc_device(sspp_ctx* ctx, int64_t ncols, const int32_t* d_dims, const int64_t* d_col_ptr,
                             const int32_t* d_rows) {
    if (!ctx) return SSPP_ERR_BAD_INPUT;
    cudaSetDevice(ctx->cfg.device);
    if (ncols < 0 || !d_col_ptr) return set_err(ctx, SSPP_ERR_BAD_INPUT, "null input array");
    // col_ptr is validated on the host: it is small next to the rows
    std::vector<int64_t> cp(size_t(ncols) + 1);
    CK(cudaMemcpy(cp.data(), d_col_ptr, sizeof(int64_t) * (ncols + 1), cudaMemcpyDeviceToHost));
    if (!validate_colptr(cp.data(), ncols)) return set_err(ctx, SSPP_ERR_BAD_INPUT, "col_ptr must start at 0 and be non-decreasing");
    const int64_t nnz = cp[size_t(ncols)];
    int rc = load_common(ctx, ncols, nnz);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    if (ncols) CK(cudaMemcpyAsync(ctx->D.in_dims, d_dims, sizeof(int32_t) * ncols, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->D.in_colptr, d_col_ptr, sizeof(int64_t) * (ncols + 1), cudaMemcpyDeviceToDevice, s));
    if (nnz) CK(cudaMemcpyAsync(ctx->D.in_rows, d_rows, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    ctx->loaded = true;
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
        if (rc != SSPP_ERR_CAPACITY || !ctx->err.empty()) return rc;
        // arena exhausted: grow it and redo the whole reduction from the input
        ctx->arena_request = std::max<int64_t>(ctx->D.arena_cap * 2, arena_need(ctx));
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
    if (n > 0 && cudaMemcpy(out, ctx->D.pairs, sizeof(int64_t) * 2 * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
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
    o->additions = c[CNT_ADDITIONS];
    o->add_ints = c[CNT_ADD_INTS];
    o->published_ints = c[CNT_PUBLISHED];
    o->displaced = c[CNT_DISPLACED];
    o->ss_steps = ctx->ss_steps;
    o->npairs = ctx->computed ? c[CNT_NPAIRS] : 0;
    o->nessential = ctx->computed ? c[CNT_NESS] : 0;
    o->init_ms = ctx->init_ms;
    o->compute_ms = ctx->compute_ms;
    return SSPP_OK;
}

}  // extern "C"
