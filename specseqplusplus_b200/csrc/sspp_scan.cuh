// Three-pass exclusive scan over an index space with a value functor and a
// sink functor: value(i) -> int64, sink(i, exclusive_prefix).  Used for column
// offsets and stream compaction.  Tiles of 4096 items per 256-thread block;
// the block sums are scanned by one block.
#pragma once
#include "sspp_kernels.cuh"

namespace sspp {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
    __shared__ int64_t warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t inc = warp_inclusive_scan(v);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int64_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
        int64_t ti = warp_inclusive_scan(t);
        if (lane < kScanThreads / 32) warp_tot[lane] = ti - t;
        if (lane == kScanThreads / 32 - 1) *total = ti;
    }
    __syncthreads();
    int64_t r = warp_tot[wid] + inc - v;
    __syncthreads();
    return r;
}

template <class F>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(F value, int64_t n, int64_t* blk) {
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    int64_t s = 0;
#pragma unroll 4
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k;
        if (i < n) s += value(i);
    }
    __shared__ int64_t tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) blk[blockIdx.x] = tot;
}

// exclusive scan of blk[0..nb) in place; blk[nb] = total
__global__ void __launch_bounds__(1024) k_scan_blocks(int64_t* blk, int64_t nb);

template <class F, class G>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(F value, G sink, int64_t n, const int64_t* blk) {
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    int64_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k;
        v[k] = (i < n) ? value(i) : 0;
        s += v[k];
    }
    __shared__ int64_t tot;
    int64_t run = block_exclusive_scan(s, &tot) + blk[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k;
        if (i < n) sink(i, run, v[k]);
        run += v[k];
    }
}

// blk must hold at least scan_blocks(n) + 1 entries.
inline int64_t scan_blocks(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

template <class F, class G>
void scan(F value, G sink, int64_t n, int64_t* blk, cudaStream_t s) {
    int64_t nb = scan_blocks(n);
    if (nb == 0) {
        cudaMemsetAsync(blk, 0, sizeof(int64_t), s);
        return;
    }
    k_scan_reduce<<<unsigned(nb), kScanThreads, 0, s>>>(value, n, blk);
    k_scan_blocks<<<1, 1024, 0, s>>>(blk, nb);
    k_scan_apply<<<unsigned(nb), kScanThreads, 0, s>>>(value, sink, n, blk);
}

}  // namespace sspp
