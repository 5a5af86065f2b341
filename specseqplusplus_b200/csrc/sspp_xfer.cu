// Staged host <-> device transfers (see sspp_xfer.h).
#include "sspp_xfer.h"

#include <algorithm>
#include <cstring>

namespace sspp {

namespace {
constexpr size_t kHalfBytes = size_t(32) << 20;    // each half of the pinned buffer
constexpr size_t kDirectBytes = size_t(1) << 20;   // below this, plain copies
constexpr size_t kMinTaskBytes = size_t(1) << 20;  // smallest share of one host thread
}  // namespace

HostPool::HostPool(int threads) {
    for (int i = 1; i < threads; i++) workers_.emplace_back([this] { loop(); });
}

HostPool::~HostPool() {
    {
        std::lock_guard<std::mutex> l(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
}

void HostPool::loop() {
    uint64_t seen = 0;
    for (;;) {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        while (next_ < tasks_) {
            const int i = next_++;
            const std::function<void(int)>* f = fn_;
            l.unlock();
            (*f)(i);
            l.lock();
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
}

void HostPool::run(int tasks, const std::function<void(int)>& fn) {
    if (tasks <= 0) return;
    if (tasks == 1 || workers_.empty()) {
        for (int i = 0; i < tasks; i++) fn(i);
        return;
    }
    std::unique_lock<std::mutex> l(mu_);
    fn_ = &fn;
    tasks_ = tasks;
    next_ = 0;
    pending_ = tasks;
    gen_++;
    cv_.notify_all();
    while (next_ < tasks_) {
        const int i = next_++;
        l.unlock();
        fn(i);
        l.lock();
        --pending_;
    }
    done_cv_.wait(l, [&] { return pending_ == 0; });
    fn_ = nullptr;
}

Xfer::~Xfer() {
    if (stage_) {
        for (int h = 0; h < 2; h++)
            if (used_[h]) cudaEventSynchronize(ev_[h]);
        cudaFreeHost(stage_);
    }
    for (auto e : ev_)
        if (e) cudaEventDestroy(e);
    delete pool_;
}

HostPool& Xfer::pool() {
    if (!pool_) {
        const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
        pool_ = new HostPool(threads_ > 0 ? std::min(threads_, int(hw)) : int(hw));
    }
    return *pool_;
}

cudaError_t Xfer::ensure() {
    if (stage_) return cudaSuccess;
    cudaError_t e = cudaMallocHost(&stage_, 2 * kHalfBytes);
    if (e != cudaSuccess) {
        stage_ = nullptr;
        return e;
    }
    half_ = kHalfBytes;
    for (int h = 0; h < 2; h++) {
        e = cudaEventCreateWithFlags(&ev_[h], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void Xfer::parallel_copy(const std::vector<Piece>& pieces, const std::vector<Seg>& segs, size_t fill,
                         uint8_t* stage, bool to_stage) {
    const int tasks = int(std::max<size_t>(1, std::min<size_t>(size_t(pool().size()), fill / kMinTaskBytes)));
    pool().run(tasks, [&](int t) {
        const size_t lo = fill * size_t(t) / size_t(tasks), hi = fill * size_t(t + 1) / size_t(tasks);
        for (const Seg& g : segs) {
            const size_t a = std::max(lo, g.so), b = std::min(hi, g.so + g.len);
            if (a >= b) continue;
            const Piece& p = pieces[g.piece];
            if (to_stage)
                std::memcpy(stage + a, static_cast<const uint8_t*>(p.src) + g.off + (a - g.so), b - a);
            else
                std::memcpy(static_cast<uint8_t*>(p.dst) + g.off + (a - g.so), stage + a, b - a);
        }
    });
}

// next chunk of at most `cap` bytes of the piece stream starting at (pi, po)
static size_t next_chunk(const std::vector<Piece>& pieces, size_t& pi, size_t& po, size_t cap,
                         std::vector<size_t>& out) {
    size_t fill = 0;
    while (pi < pieces.size() && fill < cap) {
        const size_t take = std::min(cap - fill, pieces[pi].bytes - po);
        if (take) {
            out.push_back(pi);
            out.push_back(po);
            out.push_back(take);
            out.push_back(fill);
        }
        fill += take;
        po += take;
        if (po == pieces[pi].bytes) {
            pi++;
            po = 0;
        }
    }
    return fill;
}

// host memory the copy engines can read directly (cudaMallocHost / registered)
static bool pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // unregistered pageable memory on some drivers
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static bool all_pinned(const std::vector<Piece>& pieces, bool src) {
    for (const Piece& p : pieces)
        if (p.bytes && !pinned(src ? p.src : p.dst)) return false;
    return true;
}

cudaError_t Xfer::h2d(const std::vector<Piece>& pieces, cudaStream_t s) {
    size_t total = 0;
    for (const Piece& p : pieces) total += p.bytes;
    if (total == 0) return cudaSuccess;
    cudaError_t e;
    if (total <= kDirectBytes || all_pinned(pieces, true)) {  // pinned sources: straight to the copy engine
        for (const Piece& p : pieces)
            if (p.bytes && (e = cudaMemcpyAsync(p.dst, p.src, p.bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
                return e;
        return cudaStreamSynchronize(s);  // pageable sources may be reused by the caller
    }
    if ((e = ensure()) != cudaSuccess) return e;
    size_t pi = 0, po = 0;
    int h = 0;
    std::vector<size_t> raw;
    std::vector<Seg> segs;
    for (;;) {
        raw.clear();
        const size_t fill = next_chunk(pieces, pi, po, half_, raw);
        if (fill == 0) break;
        segs.clear();
        for (size_t i = 0; i < raw.size(); i += 4) segs.push_back({raw[i], raw[i + 1], raw[i + 2], raw[i + 3]});
        if (used_[h] && (e = cudaEventSynchronize(ev_[h])) != cudaSuccess) return e;
        uint8_t* st = stage_ + size_t(h) * half_;
        parallel_copy(pieces, segs, fill, st, true);
        for (size_t k = 0; k < segs.size();) {  // one DMA per run contiguous on the device
            uint8_t* d0 = static_cast<uint8_t*>(pieces[segs[k].piece].dst) + segs[k].off;
            size_t len = segs[k].len, k2 = k + 1;
            const int grp = pieces[segs[k].piece].group;
            while (k2 < segs.size() && grp >= 0 && pieces[segs[k2].piece].group == grp &&
                   static_cast<uint8_t*>(pieces[segs[k2].piece].dst) + segs[k2].off == d0 + len)
                len += segs[k2++].len;
            if ((e = cudaMemcpyAsync(d0, st + segs[k].so, len, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
            k = k2;
        }
        if ((e = cudaEventRecord(ev_[h], s)) != cudaSuccess) return e;
        used_[h] = true;
        h ^= 1;
    }
    return cudaSuccess;
}

cudaError_t Xfer::d2h(const std::vector<Piece>& pieces, cudaStream_t s) {
    size_t total = 0;
    for (const Piece& p : pieces) total += p.bytes;
    if (total == 0) return cudaSuccess;
    cudaError_t e;
    if (total <= kDirectBytes || all_pinned(pieces, false)) {
        for (const Piece& p : pieces)
            if (p.bytes && (e = cudaMemcpyAsync(p.dst, p.src, p.bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                return e;
        return cudaStreamSynchronize(s);
    }
    if ((e = ensure()) != cudaSuccess) return e;
    size_t pi = 0, po = 0;
    int h = 0;
    std::vector<size_t> raw;
    std::vector<Seg> cur, prev;
    size_t prev_fill = 0;
    int prev_h = -1;
    for (;;) {
        raw.clear();
        const size_t fill = next_chunk(pieces, pi, po, half_, raw);
        if (fill > 0) {
            cur.clear();
            for (size_t i = 0; i < raw.size(); i += 4) cur.push_back({raw[i], raw[i + 1], raw[i + 2], raw[i + 3]});
            if (used_[h] && (e = cudaEventSynchronize(ev_[h])) != cudaSuccess) return e;
            uint8_t* st = stage_ + size_t(h) * half_;
            for (size_t k = 0; k < cur.size();) {  // one DMA per run contiguous on the device
                const uint8_t* s0 = static_cast<const uint8_t*>(pieces[cur[k].piece].src) + cur[k].off;
                size_t len = cur[k].len, k2 = k + 1;
                const int grp = pieces[cur[k].piece].group;
                while (k2 < cur.size() && grp >= 0 && pieces[cur[k2].piece].group == grp &&
                       static_cast<const uint8_t*>(pieces[cur[k2].piece].src) + cur[k2].off == s0 + len)
                    len += cur[k2++].len;
                if ((e = cudaMemcpyAsync(st + cur[k].so, s0, len, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                    return e;
                k = k2;
            }
            if ((e = cudaEventRecord(ev_[h], s)) != cudaSuccess) return e;
            used_[h] = true;
        }
        if (prev_h >= 0) {  // the previous chunk's bytes go out while this chunk's DMA runs
            if ((e = cudaEventSynchronize(ev_[prev_h])) != cudaSuccess) return e;
            parallel_copy(pieces, prev, prev_fill, stage_ + size_t(prev_h) * half_, false);
        }
        if (fill == 0) break;
        prev.swap(cur);
        prev_fill = fill;
        prev_h = h;
        h ^= 1;
    }
    return cudaSuccess;
}

}  // namespace sspp
