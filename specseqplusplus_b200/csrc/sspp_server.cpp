// Resident request loop with continuous batching (include/sspp.h, "Serving").
//
// No counterpart in the reference, whose command line reduces one file per
// process (src/main.cu:269-352).  Requests are copied (or referenced) at
// submission and queued in arrival order.  Each worker thread owns a context
// (its own stream, device buffers and pinned staging) and loops: take the
// queued requests, oldest first, while the batch's device-memory estimate
// fits the worker's share of the budget; reduce them as one block-diagonal
// batch; hand every request its own pairs and essentials.  Requests that
// arrive meanwhile wait for the next free worker, which forms the next batch
// from whatever is queued then, so batches are formed continuously and the
// workers' batches overlap on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/sspp.h"
#include "sspp_tune.h"

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { KIND_MATRIX = 0, KIND_RIPS = 1, KIND_LOWERSTAR = 2 };

struct Request {
    int64_t id = 0;
    int64_t ncols = 0, nnz = 0;       // built requests: estimates until built
    int kind = KIND_MATRIX;
    // built requests: the point cloud or field, and the builder's arguments
    std::vector<float> fin_copy;
    const float* fin = nullptr;
    int64_t g[3] = {0, 0, 0};        // Rips: points, space dimension; lower-star: grid sizes
    float radius = 0.0f;
    int32_t maxdim = 3;
    bool want_values = false;
    std::unique_ptr<float[]> values;  // the built matrix's filtration values, if asked for
    std::vector<int32_t> dims_copy;
    std::vector<int64_t> colptr_copy;
    std::vector<int32_t> rows_copy;
    const int32_t* dims = nullptr;
    const int64_t* colptr = nullptr;
    const int32_t* rows = nullptr;
    double est = 0;
    int state = SSPP_REQ_QUEUED;
    int32_t status = SSPP_OK;
    std::string msg;
    // results (uninitialised storage: filled by the staged copy's threads)
    std::unique_ptr<int64_t[]> pairs, ess;
    int64_t npairs = 0, ness = 0;
    Clock::time_point t_submit, t_done;
};

struct Phases {
    double load = 0, reduce = 0, results = 0;  // seconds
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct sspp_server {
    sspp_server_config cfg{};
    sspp_params params{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 0;
    std::vector<std::thread> workers;
    bool stop = false;
    double budget = 0, share = 0;
    std::string err;
    std::vector<double> lat_ms;
    int64_t submitted = 0, completed = 0, failed = 0, rejected = 0, batches = 0, columns = 0, batch_reqs = 0;
    bool have_first = false;
    Clock::time_point t_first, t_last;
    Phases phases;
    int64_t queued_cols = 0;  // columns of the queued requests
};

namespace {

int64_t reject(sspp_server* S, const char* why);
void take_floats(Request* r, const float* p, int64_t n, int32_t flags);
int64_t enqueue(sspp_server* S, std::unique_ptr<Request> r);

// device bytes one request adds to a batch
double estimate(const sspp_params& p, int64_t ncols, int64_t nnz) {
    const double fill = sspp::tune_fill(ncols, p.model, p.dualize, p.autotune == 2, 3.0);
    const double base = double(nnz) + 7.0 * double(ncols) + 4.0;
    double b = 128.0 * double(ncols) + 4.0 * double(nnz) + 4.0 * fill * base;
    if (p.dualize || p.autotune == 2) b += 4.0 * base;  // dual columns built behind the primal ones
    return b;
}

void set_result(Request* r, int32_t status, const char* msg) {
    r->status = status;
    r->msg = msg ? msg : "";
}

// one batch through one context; SSPP_OK when every request has its results
int32_t try_batch(sspp_ctx* ctx, const sspp_params& params, const std::vector<Request*>& b, Phases& ph) {
    if (!ctx) {
        for (Request* r : b) set_result(r, SSPP_ERR_CUDA, "no usable CUDA device");
        return SSPP_ERR_CUDA;
    }
    const int32_t k = int32_t(b.size());
    std::vector<int64_t> nc(b.size());
    std::vector<const int32_t*> d(b.size()), rw(b.size());
    std::vector<const int64_t*> cp(b.size());
    for (size_t i = 0; i < b.size(); i++) {
        nc[i] = b[i]->ncols;
        d[i] = b[i]->dims;
        cp[i] = b[i]->colptr;
        rw[i] = b[i]->rows;
    }
    const Clock::time_point t0 = Clock::now();
    int32_t rc = sspp_load_batch(ctx, k, nc.data(), d.data(), cp.data(), rw.data());
    const Clock::time_point t1 = Clock::now();
    if (rc == SSPP_OK) rc = sspp_reduce(ctx, &params, nullptr);
    const Clock::time_point t2 = Clock::now();
    ph.load += ms_between(t0, t1) / 1000.0;
    ph.reduce += ms_between(t1, t2) / 1000.0;
    if (rc != SSPP_OK) {
        for (Request* r : b) set_result(r, rc, sspp_last_error(ctx));
        return rc;
    }
    std::vector<int64_t> np(b.size()), ne(b.size());
    rc = sspp_batch_counts(ctx, np.data(), ne.data());
    std::vector<int64_t*> po(b.size()), eo(b.size());
    if (rc == SSPP_OK) {
        for (size_t i = 0; i < b.size(); i++) {
            b[i]->npairs = np[i];
            b[i]->ness = ne[i];
            b[i]->pairs.reset(new int64_t[size_t(std::max<int64_t>(2 * np[i], 1))]);
            b[i]->ess.reset(new int64_t[size_t(std::max<int64_t>(ne[i], 1))]);
            po[i] = b[i]->pairs.get();
            eo[i] = b[i]->ess.get();
        }
        rc = sspp_batch_copy(ctx, po.data(), eo.data());
    }
    ph.results += ms_between(t2, Clock::now()) / 1000.0;
    for (Request* r : b) set_result(r, rc, rc == SSPP_OK ? nullptr : sspp_last_error(ctx));
    return rc;
}

// A request given as a point cloud or a field: built on the device, reduced
// alone; pairs are indices of the built matrix.
int32_t try_built(sspp_ctx* ctx, const sspp_params& params, Request* r, Phases& ph) {
    if (!ctx) {
        set_result(r, SSPP_ERR_CUDA, "no usable CUDA device");
        return SSPP_ERR_CUDA;
    }
    const Clock::time_point t0 = Clock::now();
    int32_t rc = r->kind == KIND_RIPS
                     ? sspp_load_rips(ctx, r->g[0], int32_t(r->g[1]), r->fin, r->radius, r->maxdim)
                     : sspp_load_lowerstar(ctx, r->g[0], r->g[1], r->g[2], r->fin, r->maxdim);
    const Clock::time_point t1 = Clock::now();
    if (rc == SSPP_OK) rc = sspp_reduce(ctx, &params, nullptr);
    const Clock::time_point t2 = Clock::now();
    ph.load += ms_between(t0, t1) / 1000.0;
    ph.reduce += ms_between(t1, t2) / 1000.0;
    if (rc == SSPP_OK) rc = sspp_input_size(ctx, &r->ncols, &r->nnz);
    if (rc == SSPP_OK) {
        r->npairs = sspp_num_pairs(ctx);
        r->ness = sspp_num_essential(ctx);
        r->pairs.reset(new int64_t[size_t(std::max<int64_t>(2 * r->npairs, 1))]);
        r->ess.reset(new int64_t[size_t(std::max<int64_t>(r->ness, 1))]);
        if (r->npairs < 0 || r->ness < 0 || sspp_pairs(ctx, r->pairs.get(), r->npairs) != r->npairs ||
            sspp_essentials(ctx, r->ess.get(), r->ness) != r->ness)
            rc = SSPP_ERR_CUDA;
    }
    if (rc == SSPP_OK && r->want_values) {
        r->values.reset(new float[size_t(std::max<int64_t>(r->ncols, 1))]);
        rc = sspp_input_copy(ctx, nullptr, nullptr, nullptr, r->values.get());
    }
    ph.results += ms_between(t2, Clock::now()) / 1000.0;
    set_result(r, rc, rc == SSPP_OK ? nullptr : sspp_last_error(ctx));
    return rc;
}

// Several point-cloud and field requests built on the device one after
// another and reduced as one block-diagonal batch; pairs are indices of each
// built matrix.
int32_t try_built_batch(sspp_ctx* ctx, const sspp_params& params, const std::vector<Request*>& b, Phases& ph) {
    if (!ctx) {
        for (Request* r : b) set_result(r, SSPP_ERR_CUDA, "no usable CUDA device");
        return SSPP_ERR_CUDA;
    }
    std::vector<sspp_build_spec> specs(b.size());
    for (size_t i = 0; i < b.size(); i++) {
        const Request* r = b[i];
        sspp_build_spec& sp = specs[i];
        std::memset(&sp, 0, sizeof(sp));
        sp.kind = r->kind == KIND_RIPS ? SSPP_BUILD_RIPS : SSPP_BUILD_LOWERSTAR;
        sp.maxdim = r->maxdim;
        sp.size[0] = r->g[0];
        sp.size[1] = r->g[1];
        sp.size[2] = r->kind == KIND_RIPS ? 0 : r->g[2];
        sp.data = r->fin;
        sp.radius = r->radius;
    }
    const Clock::time_point t0 = Clock::now();
    int32_t rc = sspp_load_built_batch(ctx, int32_t(b.size()), specs.data());
    const Clock::time_point t1 = Clock::now();
    if (rc == SSPP_OK) rc = sspp_reduce(ctx, &params, nullptr);
    const Clock::time_point t2 = Clock::now();
    ph.load += ms_between(t0, t1) / 1000.0;
    ph.reduce += ms_between(t1, t2) / 1000.0;
    if (rc != SSPP_OK) {
        for (Request* r : b) set_result(r, rc, sspp_last_error(ctx));
        return rc;
    }
    std::vector<int64_t> np(b.size()), ne(b.size());
    rc = sspp_batch_counts(ctx, np.data(), ne.data());
    std::vector<int64_t*> po(b.size()), eo(b.size());
    for (size_t i = 0; rc == SSPP_OK && i < b.size(); i++) {
        Request* r = b[i];
        r->npairs = np[i];
        r->ness = ne[i];
        r->pairs.reset(new int64_t[size_t(std::max<int64_t>(2 * np[i], 1))]);
        r->ess.reset(new int64_t[size_t(std::max<int64_t>(ne[i], 1))]);
        po[i] = r->pairs.get();
        eo[i] = r->ess.get();
        const int64_t nc = sspp_batch_values(ctx, int32_t(i), nullptr, 0);
        if (nc < 0) {
            rc = SSPP_ERR_CUDA;
            break;
        }
        r->ncols = nc;
        if (r->want_values) {
            r->values.reset(new float[size_t(std::max<int64_t>(nc, 1))]);
            if (sspp_batch_values(ctx, int32_t(i), r->values.get(), nc) != nc) rc = SSPP_ERR_CUDA;
        }
    }
    if (rc == SSPP_OK) rc = sspp_batch_copy(ctx, po.data(), eo.data());
    ph.results += ms_between(t2, Clock::now()) / 1000.0;
    for (Request* r : b) set_result(r, rc, rc == SSPP_OK ? nullptr : sspp_last_error(ctx));
    return rc;
}

void worker_main(sspp_server* S, int host_threads) {
    sspp_config c;
    std::memset(&c, 0, sizeof(c));
    c.device = S->cfg.device;
    c.host_threads = host_threads;
    c.sm_share = S->cfg.workers;  // the workers' persistent reductions run side by side
    sspp_ctx* ctx = sspp_create(&c);
    const size_t max_req = S->cfg.max_batch_requests > 0 ? size_t(S->cfg.max_batch_requests) : SIZE_MAX;
    const int64_t max_cols = S->cfg.max_batch_cols > 0 ? S->cfg.max_batch_cols : INT64_MAX;
    std::vector<Request*> batch;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> l(S->mu);
            S->cv_work.wait(l, [&] { return S->stop || !S->queue.empty(); });
            if (S->queue.empty()) break;  // stopping and drained
            if (S->cfg.batch_window_ms > 0 && !S->stop && S->queue.size() < max_req) {
                S->cv_work.wait_for(l, std::chrono::duration<double, std::milli>(S->cfg.batch_window_ms),
                                    [&] { return S->stop || S->queue.size() >= max_req; });
                if (S->queue.empty()) continue;  // another worker took them
            }
            // half a fair share of the queued columns, so that every worker
            // gets two or more batches and their copies, builds and
            // reductions overlap on the device
            const int64_t share_of = 2 * int64_t(S->cfg.workers);
            const int64_t fair = (S->queued_cols + share_of - 1) / share_of;
            double est = 0;
            int64_t cols = 0;
            while (!S->queue.empty()) {
                Request* r = S->queue.front();
                // matrices batch with matrices, built requests with built ones
                if (!batch.empty() && ((r->kind == KIND_MATRIX) != (batch[0]->kind == KIND_MATRIX) ||
                                       est + r->est > S->share || cols + r->ncols > max_cols ||
                                       batch.size() >= max_req || cols >= fair))
                    break;
                S->queue.pop_front();
                S->queued_cols -= r->ncols;
                r->state = SSPP_REQ_RUNNING;
                batch.push_back(r);
                est += r->est;
                cols += r->ncols;
            }
        }
        Phases ph;
        if (batch[0]->kind != KIND_MATRIX) {
            if (batch.size() == 1) {
                try_built(ctx, S->params, batch[0], ph);
            } else {
                int32_t rc = try_built_batch(ctx, S->params, batch, ph);
                if (rc != SSPP_OK)  // isolate the request that failed
                    for (Request* r : batch) try_built(ctx, S->params, r, ph);
            }
        } else {
            int32_t rc = try_batch(ctx, S->params, batch, ph);
            if (rc != SSPP_OK && batch.size() > 1)  // isolate the request that failed
                for (Request* r : batch) try_batch(ctx, S->params, {r}, ph);
        }
        {
            std::lock_guard<std::mutex> l(S->mu);
            S->phases.load += ph.load;
            S->phases.reduce += ph.reduce;
            S->phases.results += ph.results;
            const Clock::time_point now = Clock::now();
            for (Request* r : batch) {
                r->t_done = now;
                r->state = r->status == SSPP_OK ? SSPP_REQ_DONE : SSPP_REQ_FAILED;
                if (r->status == SSPP_OK) {
                    S->completed++;
                    S->columns += r->ncols;
                    S->lat_ms.push_back(ms_between(r->t_submit, now));
                } else {
                    S->failed++;
                }
                // inputs are no longer needed
                std::vector<int32_t>().swap(r->dims_copy);
                std::vector<int64_t>().swap(r->colptr_copy);
                std::vector<int32_t>().swap(r->rows_copy);
                std::vector<float>().swap(r->fin_copy);
                r->fin = nullptr;
                r->dims = nullptr;
                r->colptr = nullptr;
                r->rows = nullptr;
            }
            S->batches++;
            S->batch_reqs += int64_t(batch.size());
            S->t_last = now;
        }
        S->cv_done.notify_all();
    }
    if (ctx) sspp_destroy(ctx);
}

Request* find(sspp_server* S, int64_t id) {
    auto it = S->reqs.find(id);
    return it == S->reqs.end() ? nullptr : it->second.get();
}

bool finished(const Request* r) { return r->state == SSPP_REQ_DONE || r->state == SSPP_REQ_FAILED; }

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const double pos = q * double(v.size() - 1);
    const size_t lo = size_t(std::floor(pos)), hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (pos - double(lo)) * (v[hi] - v[lo]);
}

}  // namespace

extern "C" {

sspp_server* sspp_server_create(const sspp_server_config* cfg, const sspp_params* params) {
    auto* S = new (std::nothrow) sspp_server;
    if (!S) return nullptr;
    if (cfg) S->cfg = *cfg;
    if (params) S->params = *params;
    else sspp_default_params(&S->params);
    if (S->cfg.workers <= 0) S->cfg.workers = 2;
    if (cudaSetDevice(S->cfg.device) != cudaSuccess) {
        delete S;
        return nullptr;
    }
    S->budget = double(S->cfg.memory_budget);
    if (S->budget <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete S;
            return nullptr;
        }
        S->budget = 0.85 * double(fr);
    }
    S->share = S->budget / double(S->cfg.workers);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int per = std::max(1, int(hw) / S->cfg.workers);
    for (int w = 0; w < S->cfg.workers; w++) S->workers.emplace_back(worker_main, S, per);
    return S;
}

void sspp_server_destroy(sspp_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> l(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto& t : S->workers) t.join();
    delete S;
}

const char* sspp_server_last_error(sspp_server* S) { return S ? S->err.c_str() : "null server"; }

int64_t sspp_server_submit(sspp_server* S, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                           const int32_t* rows, int32_t flags) {
    if (!S) return -SSPP_ERR_BAD_INPUT;
    if (ncols < 0 || !col_ptr || (ncols > 0 && !dims) || col_ptr[0] != 0 || col_ptr[ncols] < 0 ||
        (col_ptr[ncols] > 0 && !rows)) {
        std::lock_guard<std::mutex> l(S->mu);
        S->err = "bad request arrays";
        S->rejected++;
        return -SSPP_ERR_BAD_INPUT;
    }
    auto r = std::make_unique<Request>();
    r->ncols = ncols;
    r->nnz = col_ptr[ncols];
    if (flags & SSPP_SUBMIT_NOCOPY) {
        r->dims = dims;
        r->colptr = col_ptr;
        r->rows = rows;
    } else {
        r->dims_copy.assign(dims, dims + ncols);
        r->colptr_copy.assign(col_ptr, col_ptr + ncols + 1);
        r->rows_copy.assign(rows, rows + r->nnz);
        r->dims = r->dims_copy.data();
        r->colptr = r->colptr_copy.data();
        r->rows = r->rows_copy.data();
    }
    r->est = estimate(S->params, ncols, r->nnz);
    return enqueue(S, std::move(r));
}

int64_t sspp_server_submit_rips(sspp_server* S, int64_t npts, int32_t space_dim, const float* points, float radius,
                                int32_t maxdim, int32_t flags) {
    if (!S) return -SSPP_ERR_BAD_INPUT;
    if (npts < 0 || (npts > 0 && !points) || space_dim < 1 || space_dim > 3 || !(radius >= 0.0f) ||
        !std::isfinite(radius) || maxdim < 0 || maxdim > 3)
        return reject(S, "bad point cloud request");
    auto r = std::make_unique<Request>();
    r->kind = KIND_RIPS;
    r->g[0] = npts;
    r->g[1] = space_dim;
    r->radius = radius;
    r->maxdim = maxdim;
    r->want_values = (flags & SSPP_SUBMIT_VALUES) != 0;
    take_floats(r.get(), points, npts * space_dim, flags);
    // the size is known once built; for batching the queue counts the
    // columns of a complex of mean degree 24 (1 + 12 + 48 + 96 per point in 3-D)
    r->ncols = (space_dim == 3 ? 157 : 61) * npts;
    r->nnz = 4 * r->ncols;
    r->est = 0;
    return enqueue(S, std::move(r));
}

int64_t sspp_server_submit_lowerstar(sspp_server* S, int64_t gx, int64_t gy, int64_t gz, const float* values,
                                     int32_t maxdim, int32_t flags) {
    if (!S) return -SSPP_ERR_BAD_INPUT;
    if (gx < 1 || gy < 1 || gz < 1 || !values || gx > INT32_MAX || gy > INT32_MAX || gz > INT32_MAX ||
        gx * gy > INT32_MAX || gx * gy * gz > INT32_MAX || maxdim < 0 || maxdim > 3)
        return reject(S, "bad field request");
    auto r = std::make_unique<Request>();
    r->kind = KIND_LOWERSTAR;
    r->g[0] = gx;
    r->g[1] = gy;
    r->g[2] = gz;
    r->maxdim = maxdim;
    r->want_values = (flags & SSPP_SUBMIT_VALUES) != 0;
    const int64_t nv = gx * gy * gz;
    take_floats(r.get(), values, nv, flags);
    // at most 7 edges, 12 triangles and 6 tetrahedra start at each vertex
    r->ncols = 26 * nv;
    r->nnz = 74 * nv;
    r->est = estimate(S->params, r->ncols, r->nnz);
    return enqueue(S, std::move(r));
}

int64_t sspp_server_values(sspp_server* S, int64_t id, float* out, int64_t cap) {
    if (!S || cap < 0 || (!out && cap > 0)) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || r->state != SSPP_REQ_DONE || !r->values) return -1;
    const int64_t n = std::min<int64_t>(cap, r->ncols);
    if (n > 0) std::memcpy(out, r->values.get(), sizeof(float) * size_t(n));
    return r->ncols;
}

}  // extern "C"

namespace {

int64_t reject(sspp_server* S, const char* why) {
    std::lock_guard<std::mutex> l(S->mu);
    S->err = why;
    S->rejected++;
    return -SSPP_ERR_BAD_INPUT;
}

void take_floats(Request* r, const float* p, int64_t n, int32_t flags) {
    if (flags & SSPP_SUBMIT_NOCOPY) {
        r->fin = p;
    } else {
        r->fin_copy.assign(p, p + n);
        r->fin = r->fin_copy.data();
    }
}

int64_t enqueue(sspp_server* S, std::unique_ptr<Request> r) {
    std::lock_guard<std::mutex> l(S->mu);
    if (r->est > S->budget) {
        S->err = "request larger than the device-memory budget";
        S->rejected++;
        return -SSPP_ERR_CAPACITY;
    }
    const int64_t id = S->next_id++;
    r->id = id;
    r->t_submit = Clock::now();
    if (!S->have_first) {
        S->have_first = true;
        S->t_first = r->t_submit;
    }
    S->submitted++;
    S->queued_cols += r->ncols;
    S->queue.push_back(r.get());
    S->reqs.emplace(id, std::move(r));
    S->cv_work.notify_one();
    return id;
}

}  // namespace

extern "C" {

int32_t sspp_server_wait(sspp_server* S, int64_t id, double timeout_ms) {
    if (!S) return SSPP_ERR_BAD_INPUT;
    std::unique_lock<std::mutex> l(S->mu);
    if (!find(S, id)) return SSPP_ERR_STATE;
    // the request is looked up again on every wake-up: another thread may
    // release it (and free it) while this one waits with the lock released
    auto done = [&] {
        Request* r = find(S, id);
        return !r || finished(r);
    };
    if (timeout_ms < 0) S->cv_done.wait(l, done);
    else if (!S->cv_done.wait_for(l, std::chrono::duration<double, std::milli>(timeout_ms), done))
        return SSPP_ERR_TIMEOUT;
    return SSPP_OK;
}

int32_t sspp_server_state(sspp_server* S, int64_t id) {
    if (!S) return -SSPP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    return r ? r->state : -SSPP_ERR_STATE;
}

int32_t sspp_server_result(sspp_server* S, int64_t id, char* msg, int32_t msg_cap) {
    if (!S) return SSPP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || !finished(r)) return SSPP_ERR_STATE;
    if (msg && msg_cap > 0) {
        std::strncpy(msg, r->msg.c_str(), size_t(msg_cap) - 1);
        msg[msg_cap - 1] = 0;
    }
    return r->status;
}

int64_t sspp_server_num_pairs(sspp_server* S, int64_t id) {
    if (!S) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || r->state != SSPP_REQ_DONE) return -1;
    return r->npairs;
}

int64_t sspp_server_pairs(sspp_server* S, int64_t id, int64_t* out, int64_t cap) {
    if (!S || cap < 0 || (!out && cap > 0)) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || r->state != SSPP_REQ_DONE) return -1;
    const int64_t n = std::min<int64_t>(cap, r->npairs);
    if (n > 0) std::memcpy(out, r->pairs.get(), sizeof(int64_t) * 2 * size_t(n));
    return n;
}

int64_t sspp_server_num_essential(sspp_server* S, int64_t id) {
    if (!S) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || r->state != SSPP_REQ_DONE) return -1;
    return r->ness;
}

int64_t sspp_server_essentials(sspp_server* S, int64_t id, int64_t* out, int64_t cap) {
    if (!S || cap < 0 || (!out && cap > 0)) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || r->state != SSPP_REQ_DONE) return -1;
    const int64_t n = std::min<int64_t>(cap, r->ness);
    if (n > 0) std::memcpy(out, r->ess.get(), sizeof(int64_t) * size_t(n));
    return n;
}

double sspp_server_latency_ms(sspp_server* S, int64_t id) {
    if (!S) return -1;
    std::lock_guard<std::mutex> l(S->mu);
    Request* r = find(S, id);
    if (!r || !finished(r)) return -1;
    return ms_between(r->t_submit, r->t_done);
}

int32_t sspp_server_release(sspp_server* S, int64_t id) {
    if (!S) return SSPP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> l(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end() || !finished(it->second.get())) return SSPP_ERR_STATE;
    S->reqs.erase(it);
    return SSPP_OK;
}

int32_t sspp_server_get_stats(sspp_server* S, sspp_server_stats* o) {
    if (!S || !o) return SSPP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> l(S->mu);
    std::memset(o, 0, sizeof(*o));
    o->submitted = S->submitted;
    o->completed = S->completed;
    o->failed = S->failed;
    o->rejected = S->rejected;
    o->batches = S->batches;
    o->columns = S->columns;
    o->wall_s = (S->have_first && S->batches) ? ms_between(S->t_first, S->t_last) / 1000.0 : 0.0;
    o->cols_per_s = o->wall_s > 0 ? double(S->columns) / o->wall_s : 0.0;
    o->p50_ms = percentile(S->lat_ms, 0.50);
    o->p95_ms = percentile(S->lat_ms, 0.95);
    o->p99_ms = percentile(S->lat_ms, 0.99);
    o->max_ms = S->lat_ms.empty() ? 0.0 : *std::max_element(S->lat_ms.begin(), S->lat_ms.end());
    double sum = 0;
    for (double x : S->lat_ms) sum += x;
    o->mean_ms = S->lat_ms.empty() ? 0.0 : sum / double(S->lat_ms.size());
    o->mean_batch_requests = S->batches ? double(S->batch_reqs) / double(S->batches) : 0.0;
    o->load_s = S->phases.load;
    o->reduce_s = S->phases.reduce;
    o->results_s = S->phases.results;
    return SSPP_OK;
}

int32_t sspp_server_reset_stats(sspp_server* S) {
    if (!S) return SSPP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> l(S->mu);
    S->lat_ms.clear();
    S->submitted = S->completed = S->failed = S->rejected = S->batches = S->columns = S->batch_reqs = 0;
    S->have_first = false;
    S->phases = Phases();
    return SSPP_OK;
}

}  // extern "C"
