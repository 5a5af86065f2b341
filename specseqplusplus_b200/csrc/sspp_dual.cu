// Dualization: the anti-transpose of the cleared and compressed matrix, built
// in the arena behind the primal columns, with the pivot table, the column
// states, the dimensions and the per-dimension ranges carried over.
//
// Reference counterparts:
//   count / offsets / scatter     include/kernel.h:521-560 (countNonZeros,
//                                 computeOffsets, dualizeMatrixKernel)
//   per-column sort               include/specseq.h:329-332 (one thrust::sort
//                                 per column, launched from a host loop)
//   pivot and flag remap          include/kernel.h:562-580 (dualizeAuxArray)
//   dimension reversal            include/specseq.h:347-349
//   pairs mapped back             include/specseq.h:1188
// Primal row r of primal column j becomes dual row n-1-j of dual column n-1-r.
// An apparent pair (low l, column c) of the primal matrix becomes the dual
// pair (low n-1-c, column n-1-l).  Here every step is a device pass: the
// per-column sort is one warp per column (registers up to 32 entries, shared
// memory up to 1024), and the rare longer columns are sorted by one CTA with
// shared-memory chunk sorts and merge-path merges in global memory.
//
// Mode 2 (no counterpart in the reference) dualizes after the boundary
// matrix's edge columns have been reduced: the 0-dimensional pairs are known,
// the dual columns of vertices are left alone, and the dual columns of the
// edges those pairs kill are cleared.  The dual columns of dimension >= 1 only
// hold cofaces of dimension >= 2, whose columns that reduction never touched.
// On lower-star grids the dual columns of vertices carry addition chains of
// tens of thousands of steps; mode 2 avoids them while keeping the short dual
// chains of dimensions >= 1 on Rips complexes.
#include <climits>

#include "sspp_launch.h"
#include "sspp_scan.cuh"

namespace sspp {

namespace {

constexpr int kWarpSortCap = 1024;  // ints of shared memory per warp
constexpr int kSortWarps = 8;
constexpr int kLongThreads = 1024;
constexpr int kLongChunk = 8192;    // ints sorted in shared memory by the CTA

unsigned grid_of(int64_t n, int threads, int64_t maxg) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > maxg) g = maxg;
    return unsigned(g);
}

__device__ __forceinline__ int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// misc[0] = dual region base (ints into the arena, -1 when it does not fit),
// misc[1] = dual region size, misc[2] = number of long columns.
__global__ void k_dual_count(int64_t n, const int32_t* arena, const uint64_t* desc, int32_t* cnt) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t d = desc[j];
        const int32_t* c = arena + desc_off(d) + kHdr;
        const uint32_t len = desc_len(d);
        for (uint32_t k = 0; k < len; k++) atomicAdd(&cnt[n - 1 - c[k]], 1);
    }
}

__global__ void k_dual_reserve(const int64_t* total, unsigned long long* top, int64_t arena_cap, int64_t* misc,
                               int* err) {
    const int64_t base = int64_t(*top);
    if (base + *total > arena_cap) {
        misc[0] = -1;
        atomicOr(err, ERRB_CAPACITY);
        return;
    }
    misc[0] = base;
    misc[1] = *total;
    misc[2] = 0;
    *top = (unsigned long long)(base + *total);
}

// header {len, column, 0, 0} and INT32_MAX padding of every dual slot
__global__ void k_dual_layout(int64_t n, const int32_t* cnt, const int64_t* off, const int64_t* misc,
                              int32_t* arena) {
    const int64_t base = misc[0];
    if (base < 0) return;
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x) {
        const int64_t o = base + off[c];
        const int32_t len = cnt[c];
        *reinterpret_cast<int4*>(arena + o) = make_int4(len, int32_t(c), 0, 0);
        for (int64_t k = len; k < pad4(len); k++) arena[o + kHdr + k] = INT_MAX;
    }
}

// scatter: cnt[] counts down to zero as the entries land (unsorted)
__global__ void k_dual_fill(int64_t n, const uint64_t* desc, const int64_t* off, const int64_t* misc, int32_t* cnt,
                            int32_t* arena) {
    const int64_t base = misc[0];
    if (base < 0) return;
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t d = desc[j];
        const int32_t* col = arena + desc_off(d) + kHdr;
        const uint32_t len = desc_len(d);
        for (uint32_t k = 0; k < len; k++) {
            const int64_t c = n - 1 - col[k];
            const int32_t p = atomicSub(&cnt[c], 1) - 1;
            arena[base + off[c] + kHdr + p] = int32_t(n - 1 - j);
        }
    }
}

// one warp per dual column; columns longer than kWarpSortCap go to the long list
__global__ void __launch_bounds__(kSortWarps * 32) k_dual_sort(int64_t n, const int64_t* off, int64_t* misc,
                                                              int32_t* arena, int32_t* longlist) {
    __shared__ int32_t sm[kSortWarps][kWarpSortCap];
    const int64_t base = misc[0];
    if (base < 0) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t nw = int64_t(gridDim.x) * kSortWarps;
    int32_t* s = sm[w];
    for (int64_t c = int64_t(blockIdx.x) * kSortWarps + w; c < n; c += nw) {
        int32_t* hdr = arena + base + off[c];
        const int len = hdr[0];
        int32_t* data = hdr + kHdr;
        if (len <= 1) continue;
        if (len <= 32) {
            int32_t v = lane < len ? data[lane] : INT_MAX;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const int32_t o = __shfl_xor_sync(0xffffffffu, v, j);
                    const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
                    v = keep_min ? min(v, o) : max(v, o);
                }
            }
            if (lane < len) data[lane] = v;
        } else if (len <= kWarpSortCap) {
            const int p = next_pow2(len);
            for (int i = lane; i < p; i += 32) s[i] = i < len ? data[i] : INT_MAX;
            __syncwarp();
            for (int k = 2; k <= p; k <<= 1) {
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < p; i += 32) {
                        const int ixj = i ^ j;
                        if (ixj > i) {
                            const int32_t a = s[i], b = s[ixj];
                            if ((a > b) == ((i & k) == 0)) {
                                s[i] = b;
                                s[ixj] = a;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            for (int i = lane; i < len; i += 32) data[i] = s[i];
            __syncwarp();
        } else if (lane == 0) {
            const int64_t q = atomicAdd(reinterpret_cast<unsigned long long*>(&misc[2]), 1ull);
            longlist[q] = int32_t(c);
        }
    }
}

// number of entries taken from a among the first `diag` outputs of merge(a, b)
__device__ __forceinline__ int64_t merge_split(const int32_t* a, int64_t na, const int32_t* b, int64_t nb,
                                               int64_t diag) {
    int64_t lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One CTA sorts the long columns one after the other: bitonic sorts of
// kLongChunk-int chunks in shared memory, then rounds of pairwise merges
// between the column and `tmp` (at least as long as the longest column).
__global__ void __launch_bounds__(kLongThreads) k_dual_sort_long(const int64_t* off, const int64_t* misc,
                                                                 int32_t* arena, const int32_t* longlist,
                                                                 int32_t* tmp) {
    __shared__ int32_t s[kLongChunk];
    const int64_t base = misc[0];
    if (base < 0) return;
    const int64_t nlong = misc[2];
    const int t = threadIdx.x;
    for (int64_t q = 0; q < nlong; q++) {
        int32_t* hdr = arena + base + off[longlist[q]];
        const int64_t len = hdr[0];
        int32_t* data = hdr + kHdr;
        for (int64_t ch = 0; ch < len; ch += kLongChunk) {
            const int m = int(len - ch < kLongChunk ? len - ch : kLongChunk);
            const int p = next_pow2(m);
            for (int i = t; i < p; i += kLongThreads) s[i] = i < m ? data[ch + i] : INT_MAX;
            __syncthreads();
            for (int k = 2; k <= p; k <<= 1) {
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = t; i < p; i += kLongThreads) {
                        const int ixj = i ^ j;
                        if (ixj > i) {
                            const int32_t a = s[i], b = s[ixj];
                            if ((a > b) == ((i & k) == 0)) {
                                s[i] = b;
                                s[ixj] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            for (int i = t; i < m; i += kLongThreads) data[ch + i] = s[i];
            __syncthreads();
        }
        int32_t* src = data;
        int32_t* dst = tmp;
        for (int64_t w = kLongChunk; w < len; w <<= 1) {
            for (int64_t a0 = 0; a0 < len; a0 += 2 * w) {
                const int64_t na = (a0 + w < len ? w : len - a0);
                const int64_t nb = (a0 + 2 * w < len ? w : (len - a0 - na > 0 ? len - a0 - na : 0));
                const int32_t* A = src + a0;
                const int32_t* B = A + na;
                const int64_t tot = na + nb;
                const int64_t per = (tot + kLongThreads - 1) / kLongThreads;
                const int64_t o0 = int64_t(t) * per < tot ? int64_t(t) * per : tot;
                const int64_t o1 = o0 + per < tot ? o0 + per : tot;
                int64_t ia = merge_split(A, na, B, nb, o0);
                int64_t ib = o0 - ia;
                for (int64_t o = o0; o < o1; o++) {
                    if (ia < na && (ib >= nb || A[ia] <= B[ib])) dst[a0 + o] = A[ia++];
                    else dst[a0 + o] = B[ib++];
                }
            }
            __syncthreads();
            int32_t* x = src;
            src = dst;
            dst = x;
        }
        if (src != data)
            for (int64_t i = t; i < len; i += kLongThreads) data[i] = src[i];
        __syncthreads();
    }
}

// dual descriptors, lows and states; primal `state` and `pdim` are read at
// n-1-c.  h0_done: the 0-dimensional pairs came from the boundary matrix, so
// the dual columns of vertices are never reduced.
__global__ void k_dual_finish(int64_t n, const int64_t* off, const int64_t* misc, const int32_t* arena,
                              uint64_t* desc, int32_t* low, const uint8_t* pstate, const int32_t* pdim, int h0_done,
                              uint8_t* nstate) {
    const int64_t base = misc[0];
    if (base < 0) return;
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x) {
        const int64_t o = base + off[c];
        const int32_t len = arena[o];
        desc[c] = pack_desc(uint64_t(o), uint32_t(len));
        low[c] = len ? arena[o + kHdr + len - 1] : -1;
        const uint8_t ps = pstate[n - 1 - c];
        nstate[c] = ps == ST_DROPPED ? ST_DROPPED : ((len && !(h0_done && pdim[n - 1 - c] == 0)) ? ST_ACTIVE : ST_ZERO);
    }
}

// primal pairs (low l, column c) -> dual (low n-1-c, column n-1-l); the dual
// column n-1-c of the negative simplex c is cleared (twist clearing of the
// dual).  With h0_done the pairs of vertices came from reducing the boundary
// matrix's edges, so their dual owners (vertex columns) are not checked.
__global__ void k_dual_pivots(int64_t n, const uint64_t* pivot, const int64_t* off, const int64_t* misc,
                              const int32_t* low, const int32_t* pdim, int h0_done, uint64_t* npivot, uint8_t* nstate,
                              uint8_t* cleared, int* err) {
    const int64_t base = misc[0];
    if (base < 0) return;
    for (int64_t l = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; l < n; l += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t e = pivot[l];
        if (e == kNoOwner) continue;
        const int64_t dc = n - 1 - l, dr = n - 1 - pv_col(e);
        const bool vertex_owner = h0_done && pdim[l] == 0;
        if (!vertex_owner && low[dc] != dr) {  // self-check: the dual owner's lowest row
            atomicOr(err, ERRB_CHECK);
            continue;
        }
        npivot[dr] = pv_pack(int32_t(dc), uint64_t(base + off[dc]));
        nstate[dc] = vertex_owner ? ST_ZERO : ST_OWNER;
        nstate[dr] = ST_CLEARED;
        cleared[dr] = 1;
    }
}

__global__ void k_reverse_i32(int32_t* a, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n / 2; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t x = a[i];
        a[i] = a[n - 1 - i];
        a[n - 1 - i] = x;
    }
}

__global__ void k_dual_diminfo(int64_t n, DimInfo* info) {
    const int d = threadIdx.x;
    if (d < kNumDims) {
        const int32_t b = info->col_begin[d], e = info->col_end[d];
        info->col_begin[d] = int32_t(n - e);
        info->col_end[d] = int32_t(n - b);
    }
}

}  // namespace

int dualize(Device& D, int mode, cudaStream_t s) {
    const int h0_done = mode == 2;
    const int64_t n = D.n;
    const unsigned g = grid_of(n, 256, 65536);
    int32_t* cnt = D.leftmost;  // free after the init passes
    int64_t* off = D.scratch64;
    cudaMemsetAsync(cnt, 0, sizeof(int32_t) * n, s);
    k_dual_count<<<g, 256, 0, s>>>(n, D.arena, D.desc, cnt);
    scan([=] __device__(int64_t c) -> int64_t { return slot_ints(cnt[c]); },
         [=] __device__(int64_t c, int64_t pre, int64_t) { off[c] = pre; }, n, D.blk, s);
    k_dual_reserve<<<1, 1, 0, s>>>(D.blk + scan_blocks(n), D.arena_top, D.arena_cap, D.misc, D.err);
    k_dual_layout<<<g, 256, 0, s>>>(n, cnt, off, D.misc, D.arena);
    k_dual_fill<<<g, 256, 0, s>>>(n, D.desc, off, D.misc, cnt, D.arena);
    k_dual_sort<<<grid_of(n, kSortWarps, 16384), kSortWarps * 32, 0, s>>>(n, off, D.misc, D.arena, D.active);
    // the pairs buffer (4n ints) is free until the pairs are extracted
    k_dual_sort_long<<<1, kLongThreads, 0, s>>>(off, D.misc, D.arena, D.active, reinterpret_cast<int32_t*>(D.pairs));
    k_dual_finish<<<g, 256, 0, s>>>(n, off, D.misc, D.arena, D.desc, D.low, D.state, D.dim, h0_done, D.negative);
    fill_i64(reinterpret_cast<int64_t*>(D.death_of), -1, n, s);  // kNoOwner
    cudaMemsetAsync(D.cleared, 0, n, s);
    k_dual_pivots<<<g, 256, 0, s>>>(n, D.pivot, off, D.misc, D.low, D.dim, h0_done,
                                    reinterpret_cast<uint64_t*>(D.death_of), D.negative, D.cleared, D.err);
    cudaMemcpyAsync(D.pivot, D.death_of, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(D.state, D.negative, n, cudaMemcpyDeviceToDevice, s);
    k_reverse_i32<<<g, 256, 0, s>>>(D.dim, n);
    k_dual_diminfo<<<1, 32, 0, s>>>(n, D.diminfo);
    return 16;
}

}  // namespace sspp
