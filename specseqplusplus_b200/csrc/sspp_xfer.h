// Host <-> device transfers of caller-owned (pageable) arrays through a pinned
// double buffer: host threads copy chunk k+1 into one half while the DMA of
// chunk k runs from the other.  A plain cudaMemcpy from pageable memory runs at
// a fraction of the link's bandwidth and keeps one host core busy; the staged
// path fills the pinned buffer with several cores and keeps the copy engine
// busy.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace sspp {

// Fixed set of host threads running one parallel loop at a time.
class HostPool {
public:
    explicit HostPool(int threads);
    ~HostPool();
    int size() const { return int(workers_.size()) + 1; }
    // runs fn(0) .. fn(tasks-1) on the pool and the calling thread; returns when all are done
    void run(int tasks, const std::function<void(int)>& fn);

private:
    void loop();
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    int tasks_ = 0, next_ = 0, pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// One copy.  Consecutive pieces of the same group (>= 0) that are adjacent on
// the device are moved by one DMA; a group must lie inside one allocation (a
// copy may not span two stream-ordered allocations, adjacent or not).
struct Piece {
    const void* src;
    void* dst;
    size_t bytes;
    int group = -1;
};

class Xfer {
public:
    Xfer() = default;
    Xfer(const Xfer&) = delete;
    Xfer& operator=(const Xfer&) = delete;
    ~Xfer();
    // host -> device, pieces in order; returns once every host source has been
    // read (the last DMA may still run on `s`)
    cudaError_t h2d(const std::vector<Piece>& pieces, cudaStream_t s);
    // device -> host; returns when every byte has landed in host memory
    cudaError_t d2h(const std::vector<Piece>& pieces, cudaStream_t s);
    HostPool& pool();
    void set_threads(int n) { threads_ = n; }  // before the first copy; 0 = all cores

private:
    cudaError_t ensure();
    struct Seg {
        size_t piece, off, len, so;
    };
    void parallel_copy(const std::vector<Piece>& pieces, const std::vector<Seg>& segs, size_t fill, uint8_t* stage,
                       bool to_stage);
    uint8_t* stage_ = nullptr;  // pinned, two halves
    size_t half_ = 0;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool used_[2] = {false, false};
    HostPool* pool_ = nullptr;
    int threads_ = 0;
};

}  // namespace sspp
