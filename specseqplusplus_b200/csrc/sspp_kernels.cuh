// Device helpers shared by the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sspp_internal.h"

namespace sspp {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Loads that must observe another SM's release (or must not hit a stale L1
// line) go through these.
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire_u8(const uint8_t* p) {
    unsigned short v;
    asm volatile("ld.acquire.gpu.global.u8 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u8(uint8_t* p, unsigned v) {
    asm volatile("st.release.gpu.global.u8 [%0], %1;" ::"l"(p), "h"((unsigned short)v) : "memory");
}
__device__ __forceinline__ uint64_t ld_cg_u64(const uint64_t* p) {
    return (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(p));
}

__device__ __forceinline__ void cnt_add(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(kFull, v, o);
        v = w < v ? w : v;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(kFull, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// inclusive warp scan
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T w = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += w;
    }
    return v;
}

}  // namespace sspp
