// Allocation-free reduction: sspp_reduce_noalloc (declared in include/sspp.h).
//
// Some callers cannot let a library allocate device memory.  A serving process
// that reserves all of its GPU memory up front for its own request pool has no
// room for, and no wish for, allocations it does not control; a pipeline that
// keeps several streams busy cannot afford cudaMalloc / cudaFree, which
// synchronise the whole device and stall every stream while they run.  The
// context API (sspp_create / sspp_reduce) allocates its buffers on first use,
// so such callers get this one entry point instead.
//
// Everything it needs lives in g_scratch below, a file-scope device array of
// kScratchInts ints (64 MiB) that every GPU which loads this library holds
// until the process exits.  The caller passes the boundary matrix and the
// output buffers, all in device memory; nothing else is allocated.  Limits:
// at most kMaxCols columns, and 3 * ncols + nnz + fill-in must fit in the
// array (the host rejects inputs that leave less than kFillReserve ints for
// fill-in; a reduction whose fill-in still overflows returns
// SSPP_ERR_CAPACITY).
//
// The array's device address is looked up with cudaGetSymbolAddress the
// first time the entry point runs on a device (with that device current) and
// cached per device, so the first call on each device should be made before
// any stream capture begins.  Every call then copies the kernel's status word
// back to the host and synchronises the stream, so it returns only once the
// reduction has finished.  Every call reuses the same array and leaves its
// contents behind; the kernel clears what must start empty (the pivot table,
// the arena cursor, the error word) itself.  Two calls that overlap on the
// GPU - on two streams, or from two threads - share the array and corrupt each
// other: serialise them.
//
// Validation happens in the kernel before any reduction: col_ptr must start
// at 0, end at nnz and never decrease (every column's range inside [0, nnz]),
// dimensions must lie in 0..7, and each column's faces must be ascending, in
// range and one dimension lower; anything else is SSPP_ERR_BAD_INPUT.
//
// The reduction is the standard twist (clearing) reduction, dimensions from
// high to low, run by one thread block: columns one after another, each
// addition a block-wide merge of two sorted index lists.  It is meant for
// modest matrices; large ones belong on the context API.
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/sspp.h"

namespace {

constexpr int64_t kScratchInts = int64_t(16) << 20;  // 64 MiB
constexpr int64_t kMaxCols = int64_t(1) << 20;
constexpr int64_t kFillReserve = int64_t(4) << 20;   // ints kept free for fill-in
constexpr int kCtl = 16;                            // control words at the start of the array
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;
constexpr int kMaxDim = 7;                          // dimensions 0..7, as the context API

// control words
enum { C_ERR = 0, C_TOP_LO = 1, C_TOP_HI = 2, C_NPAIRS_LO = 3, C_NPAIRS_HI = 4, C_MAXDIM = 5 };
enum { E_BAD_INPUT = 1, E_CAPACITY = 2 };

static __device__ __align__(256) int32_t g_scratch[kScratchInts];

void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

// block-wide exclusive prefix of v; tot = block total (two barriers)
__device__ int block_prefix(int v, int& tot, int* sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) sm[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int c = lane < kThreads / 32 ? sm[lane] : 0;
        int ci = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, ci, o);
            if (lane >= o) ci += t;
        }
        if (lane < kThreads / 32) sm[lane] = ci - c;
        if (lane == kThreads / 32 - 1) sm[kThreads / 32] = ci;
    }
    __syncthreads();
    tot = sm[kThreads / 32];
    int r = sm[wid] + inc - v;
    __syncthreads();
    return r;
}

__device__ int lower_bound_g(const int32_t* a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// out = a xor b; returns the output length
__device__ int block_xor(const int32_t* a, int na, const int32_t* b, int nb, int32_t* out, int* sm) {
    int ca = 0, cb = 0;
    const int n = na > nb ? na : nb;
    for (int base = 0; base < n; base += kThreads) {
        const int i = base + threadIdx.x;
        const bool va = i < na, vb = i < nb;
        const int x = va ? a[i] : 0, y = vb ? b[i] : 0;
        const int ra = va ? lower_bound_g(b, nb, x) : 0;
        const int rb = vb ? lower_bound_g(a, na, y) : 0;
        const bool ea = va && ra < nb && b[ra] == x;
        const bool eb = vb && rb < na && a[rb] == y;
        int ta, tb;
        const int pa = block_prefix(ea ? 1 : 0, ta, sm);
        const int pb = block_prefix(eb ? 1 : 0, tb, sm);
        if (va && !ea) out[i + ra - 2 * (ca + pa)] = x;
        if (vb && !eb) out[i + rb - 2 * (cb + pb)] = y;
        ca += ta;
        cb += tb;
    }
    __syncthreads();
    return na + nb - 2 * ca;
}

// Scratch layout (ints): [0, kCtl) control, pivot[n] (owner column of each
// row, -1 = none), off[n] and len[n] (current version of each column), then
// the arena: the input columns, followed by column versions created by
// additions.
__global__ void __launch_bounds__(kThreads) k_reduce_noalloc(int32_t* S, int64_t n, int64_t nnz, const int32_t* dims,
                                                            const int64_t* col_ptr, const int32_t* rows,
                                                            int64_t* pairs, int64_t* npairs) {
    __shared__ int sm[kThreads / 32 + 1];
    __shared__ int s_flag;
    int32_t* ctl = S;
    int32_t* pivot = S + kCtl;
    int32_t* off = pivot + n;
    int32_t* len = off + n;
    int32_t* arena = len + n;
    const int64_t arena_cap = kScratchInts - (kCtl + 3 * n);
    // what must start empty: error word, cursor, pivot table
    if (threadIdx.x == 0) {
        ctl[C_ERR] = 0;
        ctl[C_MAXDIM] = 0;
        s_flag = 0;
    }
    __syncthreads();
    if (col_ptr[0] != 0 || col_ptr[n] != nnz) {
        if (threadIdx.x == 0) ctl[C_ERR] = E_BAD_INPUT;
        return;
    }
    int maxd = 0;
    for (int64_t j = threadIdx.x; j < n; j += kThreads) {
        pivot[j] = -1;
        const int64_t b = col_ptr[j], e = col_ptr[j + 1];
        const int d = dims[j];
        // every column's range must lie inside [0, nnz] before any entry is
        // read or copied (the copy runs in the same pass as the checks)
        bool bad = b < 0 || e < b || e > nnz || d < 0 || d > kMaxDim;
        for (int64_t k = b; k < e && !bad; k++) {
            const int32_t r = rows[k];
            if (r < 0 || r >= n || (k > b && r <= rows[k - 1]) || dims[r] != d - 1) bad = true;
            else arena[k] = r;
        }
        if (bad) atomicOr(&s_flag, E_BAD_INPUT);
        off[j] = int32_t(b);
        len[j] = bad ? 0 : int32_t(e - b);
        maxd = d > maxd ? d : maxd;
    }
    atomicMax(&ctl[C_MAXDIM], maxd);
    __syncthreads();
    if (s_flag) {
        if (threadIdx.x == 0) ctl[C_ERR] = s_flag;
        return;
    }
    const int top_dim = ctl[C_MAXDIM];
    int64_t top = nnz;  // arena cursor (same value in every thread)
    for (int d = top_dim; d >= 1; d--) {
        for (int64_t j = 0; j < n; j++) {
            if (dims[j] != d || len[j] == 0) continue;  // other dimension, zero or cleared
            int32_t* w = arena + off[j];
            int wl = len[j];
            bool failed = false;
            while (wl > 0) {
                const int L = w[wl - 1];
                const int p = pivot[L];
                if (p < 0) break;
                const int32_t* pb = arena + off[p];
                const int pl = len[p];
                if (top + wl + pl > arena_cap) { failed = true; break; }
                int32_t* o = arena + top;
                const int ol = block_xor(w, wl, pb, pl, o, sm);
                top += wl + pl;
                w = o;
                wl = ol;
            }
            if (failed) {
                if (threadIdx.x == 0) ctl[C_ERR] = E_CAPACITY;
                return;
            }
            if (threadIdx.x == 0) {
                off[j] = int32_t(w - arena);
                len[j] = wl;
                if (wl > 0) {
                    const int L = w[wl - 1];
                    pivot[L] = int32_t(j);
                    len[L] = 0;  // twist: the column of the lowest row is positive
                }
            }
            __syncthreads();
        }
    }
    // pairs in birth order: row r owned by column c is the pair (r, c)
    int64_t written = 0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t r = base + threadIdx.x;
        const int c = r < n ? pivot[r] : -1;
        int tot;
        const int pre = block_prefix(c >= 0 ? 1 : 0, tot, sm);
        if (c >= 0) {
            pairs[2 * (written + pre)] = r;
            pairs[2 * (written + pre) + 1] = c;
        }
        written += tot;
    }
    if (threadIdx.x == 0) {
        *npairs = written;
        ctl[C_TOP_LO] = int32_t(top & 0xffffffff);
        ctl[C_TOP_HI] = int32_t(top >> 32);
    }
}

int32_t fail(char* msg, int32_t cap, int32_t code, const char* text) {
    if (msg && cap > 0) {
        std::strncpy(msg, text, size_t(cap) - 1);
        msg[cap - 1] = '\0';
    }
    return code;
}

}  // namespace

extern "C" int32_t sspp_reduce_noalloc(int64_t ncols, int64_t nnz, const int32_t* d_dims, const int64_t* d_col_ptr,
                                       const int32_t* d_rows, int64_t* d_pairs, int64_t* d_npairs, void* stream,
                                       char* err_msg, int32_t err_cap) {
    if (ncols < 0 || nnz < 0 || !d_col_ptr || !d_npairs || (ncols > 0 && (!d_dims || !d_pairs)) || (nnz > 0 && !d_rows))
        return fail(err_msg, err_cap, SSPP_ERR_BAD_INPUT, "null pointer or negative size");
    if (ncols > kMaxCols)
        return fail(err_msg, err_cap, SSPP_ERR_BAD_INPUT, "too many columns for the allocation-free path (max 1048576)");
    if (kCtl + 3 * ncols + nnz + kFillReserve > kScratchInts)
        return fail(err_msg, err_cap, SSPP_ERR_BAD_INPUT,
                    "matrix too large for the allocation-free path: 3 * ncols + nnz must stay below 12582896");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(err_msg, err_cap, SSPP_ERR_CUDA, "no current CUDA device");
    void* addr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            // once per device, with that device current
            cudaError_t e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_scratch);
            if (e != cudaSuccess) {
                g_scratch_addr[dev] = nullptr;
                return fail(err_msg, err_cap, SSPP_ERR_CUDA, cudaGetErrorString(e));
            }
        }
        addr = g_scratch_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_reduce_noalloc<<<1, kThreads, 0, s>>>(static_cast<int32_t*>(addr), ncols, nnz, d_dims, d_col_ptr, d_rows,
                                            d_pairs, d_npairs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(err_msg, err_cap, SSPP_ERR_CUDA, cudaGetErrorString(e));
    int32_t err = 0;
    e = cudaMemcpyAsync(&err, addr, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(err_msg, err_cap, SSPP_ERR_CUDA, cudaGetErrorString(e));
    if (err & E_BAD_INPUT)
        return fail(err_msg, err_cap, SSPP_ERR_BAD_INPUT,
                    "malformed boundary matrix (col_ptr, face order, range or dimension)");
    if (err & E_CAPACITY)
        return fail(err_msg, err_cap, SSPP_ERR_CAPACITY, "fill-in exceeded the 64 MiB allocation-free scratch array");
    return fail(err_msg, err_cap, SSPP_OK, "");
}
