// Dimension reorder, init passes, active lists and pair extraction.
//
// Reference counterparts:
//   dimension-stable reorder           include/specseq.h:439-483 (Formatted)
//   lowest one / leftmost column       include/kernel.h:444-457 (initleft_kernel)
//   apparent pivots, youngest-facet
//   clearing, negative columns         include/kernel.h:459-481 (initlookup_kernel)
//   clearing                           include/kernel.h:483-493 (clearing_kernel)
//   row compression                    include/kernel.h:495-520 (compress_kernel)
//   active list and per-dim bounds     include/specseq.h:365-409 (ColumnShrink)
//   pairs in input indices, sorted     include/specseq.h:1182-1193
// Here the reorder, the padded column layout and the compaction are device
// passes (the reference does them on the host), the active list is a device
// stream compaction, and pairs come out sorted by construction (each simplex is
// the birth of at most one pair, so compaction in birth order sorts them).
#include <climits>

#include "sspp_launch.h"
#include "sspp_scan.cuh"

namespace sspp {

__global__ void __launch_bounds__(1024) k_scan_blocks(int64_t* blk, int64_t nb) {
    __shared__ int64_t wt[32];
    __shared__ int64_t carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += 1024) {
        int64_t i = base + tid;
        int64_t v = i < nb ? blk[i] : 0;
        int64_t inc = warp_inclusive_scan(v);
        if (lane == 31) wt[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            int64_t t = wt[lane];
            int64_t ti = warp_inclusive_scan(t);
            wt[lane] = ti - t;
        }
        __syncthreads();
        int64_t ex = carry + wt[wid] + inc - v;
        if (i < nb) blk[i] = ex;
        __syncthreads();
        if (tid == 1023) carry = ex + v;
        __syncthreads();
    }
    if (tid == 0) blk[nb] = carry;
}

template <typename T>
__global__ void k_fill(T* p, T v, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) p[i] = v;
}

static unsigned grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > (int64_t(1) << 30)) g = int64_t(1) << 30;
    return unsigned(g);
}

void fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t s) {
    if (n > 0) k_fill<int32_t><<<grid_for(n, 256) > 4096 ? 4096 : grid_for(n, 256), 256, 0, s>>>(p, v, n);
}
void fill_i64(int64_t* p, int64_t v, int64_t n, cudaStream_t s) {
    if (n > 0) k_fill<int64_t><<<grid_for(n, 256) > 4096 ? 4096 : grid_for(n, 256), 256, 0, s>>>(p, v, n);
}

// Input validation before any index is used: dimensions in range and col_ptr
// non-decreasing from 0 (device-resident inputs are only checked here).  Also
// counts the columns of each dimension (dimtot, zeroed before), which give
// the host the reordered dimension ranges with the same read as the error word.
__global__ void __launch_bounds__(256) k_validate(const int32_t* dims, const int64_t* colptr, int64_t n, int* err,
                                                  unsigned long long* dimtot) {
    __shared__ unsigned s_cnt[kNumDims];
    if (threadIdx.x < kNumDims) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int64_t b0 = blockIdx.x * int64_t(blockDim.x); b0 < n; b0 += int64_t(gridDim.x) * blockDim.x) {
        const int64_t j = b0 + threadIdx.x;
        int d = -1;
        if (j < n) {
            d = dims[j];
            const int64_t a = colptr[j], b = colptr[j + 1];
            if (d < 0 || d > kMaxDim || b < a || b - a > kMaxColLen || (j == 0 && a != 0))
                atomicOr(err, ERRB_BAD_INPUT);
        }
#pragma unroll
        for (int q = 0; q < kNumDims; q++) {
            const unsigned m = __ballot_sync(kFull, d == q);
            if (lane == 0 && m) atomicAdd(&s_cnt[q], unsigned(__popc(m)));
        }
    }
    __syncthreads();
    if (threadIdx.x < kNumDims && s_cnt[threadIdx.x])
        atomicAdd(dimtot + threadIdx.x, (unsigned long long)s_cnt[threadIdx.x]);
}

int validate(Device& D, cudaStream_t s) {
    if (D.n <= 0) return 0;
    cudaMemsetAsync(D.dimtot, 0, sizeof(unsigned long long) * kNumDims, s);
    k_validate<<<grid_for(D.n, 256) > 4096 ? 4096 : grid_for(D.n, 256), 256, 0, s>>>(D.in_dims, D.in_colptr, D.n, D.err,
                                                                                     D.dimtot);
    return 1;
}

// Batch of k complexes copied side by side: complex i's face indices are
// shifted by its first column cstart[i], and its col_ptr entries (without the
// leading 0) by its first entry estart[i].
__device__ __forceinline__ int32_t batch_member(const int64_t* start, int32_t k, int64_t x) {
    int32_t a = 0, b = k;  // largest a with start[a] <= x
    while (b - a > 1) {
        const int32_t m = (a + b) >> 1;
        if (start[m] <= x) a = m;
        else b = m;
    }
    return a;
}

__global__ void k_batch_rebase(int64_t n, int64_t nnz, int32_t k, const int64_t* cstart, const int64_t* estart,
                               int64_t* colptr, int32_t* rows, int* bad) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nnz; t += stride) {
        const int32_t i = batch_member(estart, k, t);
        const int32_t r = rows[t];
        if (r < 0 || r >= cstart[i + 1] - cstart[i]) *bad = 1;  // a face outside its own complex
        rows[t] = r + int32_t(cstart[i]);
    }
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += stride)
        colptr[j + 1] += estart[batch_member(cstart, k, j)];
}

int batch_rebase(int64_t n, int64_t nnz, int32_t k, const int64_t* d_cstart, const int64_t* d_estart,
                 int64_t* colptr, int32_t* rows, int* d_bad, cudaStream_t s) {
    const int64_t m = n > nnz ? n : nnz;
    if (m == 0 || k <= 1) return 0;
    k_batch_rebase<<<grid_for(m, 256) > 16384 ? 16384 : grid_for(m, 256), 256, 0, s>>>(n, nnz, k, d_cstart, d_estart,
                                                                                       colptr, rows, d_bad);
    return 1;
}

// Per-complex result slices of a batch: the sorted pairs (by birth) and the
// ascending essentials of complex i start at the first entry >= cstart[i].
__global__ void k_batch_bounds(int32_t k, const int64_t* cstart, int64_t npairs, const int64_t* pairs, int64_t ness,
                               const int64_t* ess, int64_t* pstart, int64_t* estart) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= k; i += gridDim.x * blockDim.x) {
        const int64_t x = cstart[i];
        int64_t lo = 0, hi = npairs;
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (pairs[2 * m] < x) lo = m + 1;
            else hi = m;
        }
        pstart[i] = lo;
        lo = 0;
        hi = ness;
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (ess[m] < x) lo = m + 1;
            else hi = m;
        }
        estart[i] = lo;
    }
}

// pairs and essentials in their own complex's indices
__global__ void k_batch_localize(int64_t npairs, int64_t ness, int32_t k, const int64_t* cstart, const int64_t* pairs,
                                 const int64_t* ess, int64_t* lpairs, int64_t* less) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < npairs; t += stride) {
        const int64_t b = pairs[2 * t], o = cstart[batch_member(cstart, k, b)];
        lpairs[2 * t] = b - o;
        lpairs[2 * t + 1] = pairs[2 * t + 1] - o;
    }
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ness; t += stride)
        less[t] = ess[t] - cstart[batch_member(cstart, k, ess[t])];
}

int batch_bounds(int32_t k, const int64_t* d_cstart, int64_t npairs, const int64_t* pairs, int64_t ness,
                 const int64_t* ess, int64_t* d_pstart, int64_t* d_estart, cudaStream_t s) {
    k_batch_bounds<<<grid_for(int64_t(k) + 1, 128), 128, 0, s>>>(k, d_cstart, npairs, pairs, ness, ess, d_pstart,
                                                                 d_estart);
    return 1;
}

int batch_localize(int64_t npairs, int64_t ness, int32_t k, const int64_t* d_cstart, const int64_t* pairs,
                   const int64_t* ess, int64_t* lpairs, int64_t* less, cudaStream_t s) {
    const int64_t m = npairs > ness ? npairs : ness;
    if (m == 0) return 0;
    k_batch_localize<<<grid_for(m, 256) > 16384 ? 16384 : grid_for(m, 256), 256, 0, s>>>(npairs, ness, k, d_cstart,
                                                                                         pairs, ess, lpairs, less);
    return 1;
}

// ------------------------------------------------------------------ reorder
constexpr int kPartThreads = 256;

// per-block count of columns of each dimension; flags dims out of range
__global__ void __launch_bounds__(kPartThreads) k_dim_count(const int32_t* dims, int64_t n, int32_t* dimcnt, int* err) {
    __shared__ int cnt[kNumDims];
    if (threadIdx.x < kNumDims) cnt[threadIdx.x] = 0;
    __syncthreads();
    int64_t j = int64_t(blockIdx.x) * kPartThreads + threadIdx.x;
    if (j < n) {
        int d = dims[j];
        if (d < 0 || d > kMaxDim) atomicOr(err, ERRB_BAD_INPUT);
        else atomicAdd(&cnt[d], 1);
    }
    __syncthreads();
    if (threadIdx.x < kNumDims) dimcnt[int64_t(blockIdx.x) * kNumDims + threadIdx.x] = cnt[threadIdx.x];
}

// one block per dimension: exclusive scan of that dimension's per-block
// counts; the dimension's total goes to col_end[d] until k_dim_starts
__global__ void __launch_bounds__(1024) k_dim_offsets(int32_t* dimcnt, int64_t nb, DimInfo* info) {
    __shared__ int64_t wt[32];
    __shared__ int64_t carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, d = blockIdx.x;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += 1024) {
        int64_t i = base + tid;
        int64_t v = i < nb ? dimcnt[i * kNumDims + d] : 0;
        int64_t inc = warp_inclusive_scan(v);
        if (lane == 31) wt[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            int64_t t = wt[lane];
            int64_t ti = warp_inclusive_scan(t);
            wt[lane] = ti - t;
        }
        __syncthreads();
        int64_t ex = carry + wt[wid] + inc - v;
        if (i < nb) dimcnt[i * kNumDims + d] = int32_t(ex);
        __syncthreads();
        if (tid == 1023) carry = ex + v;
        __syncthreads();
    }
    if (tid == 0) info->col_end[d] = int32_t(carry);
}

// per-dimension totals -> dimension ranges of the reordered columns
__global__ void k_dim_starts(DimInfo* info) {
    if (threadIdx.x == 0) {
        int32_t s = 0;
        for (int d = 0; d < kNumDims; d++) {
            const int32_t c = info->col_end[d];
            info->col_begin[d] = s;
            s += c;
            info->col_end[d] = s;
        }
    }
}

// stable rank of each column inside its dimension -> reordered index
// Also starts the init passes' per-column state of reordered column idx: no
// leftmost column yet, no pivot owner, not cleared, not negative; and records
// its length (rlen, read in this kernel's coalesced pass over col_ptr, so the
// slot scan that follows reads it in reordered order without gathers).
__global__ void __launch_bounds__(kPartThreads) k_dim_assign(const int32_t* dims, const int64_t* colptr, int64_t n,
                                                             const int32_t* dimcnt, const DimInfo* info,
                                                             int32_t* newidx, int32_t* perm, int32_t* rdim,
                                                             int32_t* rlen, int32_t* leftmost, uint64_t* pivot,
                                                             uint8_t* cleared, uint8_t* negative) {
    __shared__ int wcnt[kPartThreads / 32][kNumDims];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t j = int64_t(blockIdx.x) * kPartThreads + threadIdx.x;
    int d = (j < n) ? dims[j] : -1;
    if (d > kMaxDim) d = -1;
    unsigned my_ballot = 0;
#pragma unroll
    for (int v = 0; v < kNumDims; v++) {
        unsigned b = __ballot_sync(kFull, d == v);
        if (d == v) my_ballot = b;
        if (lane == 0) wcnt[wid][v] = __popc(b);
    }
    __syncthreads();
    if (d >= 0) {
        int r = __popc(my_ballot & lanemask_lt());
        for (int w = 0; w < wid; w++) r += wcnt[w][d];
        int32_t idx = info->col_begin[d] + dimcnt[int64_t(blockIdx.x) * kNumDims + d] + r;
        newidx[j] = idx;
        perm[idx] = int32_t(j);
        rdim[idx] = d;
        const int64_t len = colptr[j + 1] - colptr[j];  // validated: 0 <= len <= kMaxColLen
        rlen[idx] = int32_t(len < 0 ? 0 : (len > kMaxColLen ? kMaxColLen : len));
        leftmost[idx] = INT_MAX;
        pivot[idx] = kNoOwner;
        cleared[idx] = 0;
        negative[idx] = 0;
    }
}

// Copies input column j into the padded arena slot of its reordered index
// i = newidx[j] with rows remapped to reordered indices; validates range,
// strict order and face dimension (a face of a dimension-d column must land in
// the reordered range of dimension d-1).  Threads walk the input columns, so
// col_ptr and the faces are read in order and each slot is written whole.
// With `lows` it also does the first init pass (include/kernel.h:444-457):
// the column's lowest row, and each row's leftmost column by atomicMin (the
// stable reorder keeps a column's rows ascending).
__global__ void k_scatter_cols(int64_t n, const int64_t* colptr, const int32_t* rows, const int32_t* dims,
                               const int32_t* newidx, const int64_t* off, const DimInfo* info, int32_t* arena,
                               uint64_t* desc, int32_t* low, int32_t* leftmost, bool lows, int* err) {
    __shared__ int32_t s_beg[kNumDims], s_end[kNumDims];
    if (threadIdx.x < kNumDims) {
        s_beg[threadIdx.x] = info->col_begin[threadIdx.x];
        s_end[threadIdx.x] = info->col_end[threadIdx.x];
    }
    __syncthreads();
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = colptr[j], e = colptr[j + 1];
        const int64_t len = e - b;
        const int32_t i = newidx[j];
        const int64_t o = off[i];
        const int dj = dims[j];
        const int32_t fb = dj > 0 ? s_beg[dj - 1] : 0, fe = dj > 0 ? s_end[dj - 1] : 0;
        bool bad = len < 0 || len > kMaxColLen;
        int32_t prev = -1, last = -1;
        int32_t* data = arena + o + kHdr;
        for (int64_t k = 0; k < len && !bad; k++) {
            const int32_t r = rows[b + k];
            if (r < 0 || r >= n || r <= prev) { bad = true; break; }
            const int32_t x = newidx[r];
            if (x < fb || x >= fe) { bad = true; break; }
            prev = r;
            data[k] = x;
            last = x;
        }
        if (bad) {
            atomicOr(err, ERRB_BAD_INPUT);
            desc[i] = pack_desc(uint64_t(o), 0);
            *reinterpret_cast<int4*>(arena + o) = make_int4(0, int32_t(i), 0, 0);
            if (lows) low[i] = -1;
        } else {
            for (int64_t k = len; k < pad4(len); k++) data[k] = INT_MAX;
            desc[i] = pack_desc(uint64_t(o), uint32_t(len));
            *reinterpret_cast<int4*>(arena + o) = make_int4(int32_t(len), int32_t(i), 0, 0);
            if (lows) {
                low[i] = len ? last : -1;
                for (int64_t k = 0; k < len; k++) atomicMin(&leftmost[data[k]], int32_t(i));
            }
        }
    }
}

int64_t reorder_total_slot(const Device& D) { return scan_blocks(D.n); }

int reorder(Device& D, bool lows, cudaStream_t s, cudaEvent_t assigned) {
    const int64_t n = D.n;
    const int64_t nb = (n + kPartThreads - 1) / kPartThreads;
    k_dim_count<<<unsigned(nb), kPartThreads, 0, s>>>(D.in_dims, n, D.dimcnt, D.err);
    k_dim_offsets<<<kNumDims, 1024, 0, s>>>(D.dimcnt, nb, D.diminfo);
    k_dim_starts<<<1, 32, 0, s>>>(D.diminfo);
    // the active list is built later: until then its buffer holds the reordered lengths
    int32_t* rlen = D.active;
    k_dim_assign<<<unsigned(nb), kPartThreads, 0, s>>>(D.in_dims, D.in_colptr, n, D.dimcnt, D.diminfo, D.newidx,
                                                       D.perm, D.dim, rlen, D.leftmost, D.pivot, D.cleared,
                                                       D.negative);
    if (assigned) cudaEventRecord(assigned, s);
    // padded column offsets in reordered order
    int64_t* off = D.scratch64;
    scan([=] __device__(int64_t i) -> int64_t { return slot_ints(rlen[i]); },
         [=] __device__(int64_t i, int64_t pre, int64_t) { off[i] = pre; }, n, D.blk, s);
    k_scatter_cols<<<grid_for(n, 256) > 65536 ? 65536 : grid_for(n, 256), 256, 0, s>>>(
        n, D.in_colptr, D.in_rows, D.in_dims, D.newidx, off, D.diminfo, D.arena, D.desc, D.low, D.leftmost, lows,
        D.err);
    return 8;
}

// ------------------------------------------------------------- init passes
// lowest row and leftmost columns when the reorder did not compute them (an
// edge collapse emptied columns in between); leftmost starts at INT_MAX
__global__ void k_init_low(int64_t n, const int32_t* arena, const uint64_t* desc, int32_t* low, int32_t* leftmost) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint64_t d = desc[i];
        const int32_t* c = arena + desc_off(d) + kHdr;
        uint32_t len = desc_len(d);
        low[i] = len ? c[len - 1] : -1;
        for (uint32_t k = 0; k < len; k++) atomicMin(&leftmost[c[k]], int32_t(i));
    }
}

__global__ void k_init_apparent(int64_t n, const int32_t* arena, const uint64_t* desc, const int32_t* low,
                                const int32_t* leftmost, uint64_t* pivot, uint8_t* cleared, uint8_t* negative,
                                long long* counters) {
    long long app = 0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        int32_t l = low[i];
        if (l < 0) continue;
        cleared[l] = 1;  // the youngest facet of any simplex is positive
        uint64_t d = desc[i];
        if (leftmost[l] == int32_t(i)) {
            pivot[l] = pv_pack(int32_t(i), desc_off(d));  // no earlier column can ever reach row l
            app++;
        }
        const int32_t* c = arena + desc_off(d) + kHdr;
        uint32_t len = desc_len(d);
        for (uint32_t k = 0; k < len; k++)
            if (leftmost[c[k]] == int32_t(i)) { negative[i] = 1; break; }
    }
    app = warp_sum(app);
    if ((threadIdx.x & 31) == 0 && app) cnt_add(&counters[CNT_APPARENT], app);
}

// Clears positive columns and removes negative rows in place.  With `app` it
// also writes the inline apparent columns (Device::app): a column that owns its
// lowest row l by an apparent pair writes app[l]; a row without an owner
// writes its own entry (each row's entry has exactly one writer).  With
// `rinfo` (non-null: the reordered dimensions) it also gathers the per-
// dimension row bounds of the schedule (min first row over non-empty columns,
// max lowest row + 1 over active ones; ColumnShrink, include/specseq.h:374-398)
// into info, whose bounds must start at INT_MAX / -1.
__global__ void k_init_compress(int64_t cb, int64_t n, int32_t* arena, uint64_t* desc, int32_t* low, const uint64_t* pivot,
                                const uint8_t* cleared, const uint8_t* negative, uint8_t* state,
                                const uint8_t* dropped, bool keep_rows, int4* app, const int32_t* rinfo,
                                DimInfo* info, long long* counters, int* err) {
    __shared__ int smin[kNumDims], smax[kNumDims];
    if (threadIdx.x < kNumDims) {
        smin[threadIdx.x] = INT_MAX;
        smax[threadIdx.x] = -1;
    }
    __syncthreads();
    long long ncl = 0, nact = 0;
    for (int64_t i = cb + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        if (app && pivot[i] == kNoOwner) app[i] = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
        uint64_t d = desc[i];
        int32_t* hdr = arena + desc_off(d);
        int32_t* c = hdr + kHdr;
        uint32_t len = desc_len(d);
        if (dropped && dropped[i]) {
            desc[i] = pack_desc(desc_off(d), 0);
            hdr[0] = 0;
            low[i] = -1;
            state[i] = ST_DROPPED;
            continue;
        }
        if (cleared[i]) {
            if (len && pv_col(pivot[low[i]]) == int32_t(i)) atomicOr(err, ERRB_BAD_INPUT);  // positive and negative
            desc[i] = pack_desc(desc_off(d), 0);
            hdr[0] = 0;
            low[i] = -1;
            state[i] = ST_CLEARED;
            ncl++;
            continue;
        }
        uint32_t m = 0;
        if (keep_rows) {
            m = len;
        } else {
            for (uint32_t k = 0; k < len; k++) {
                int32_t r = c[k];
                if (!negative[r]) c[m++] = r;
            }
        }
        for (uint32_t k = m; k < len; k++) c[k] = INT_MAX;
        desc[i] = pack_desc(desc_off(d), m);
        hdr[0] = int32_t(m);
        int32_t l = m ? c[m - 1] : -1;
        low[i] = l;
        uint8_t st = (m == 0) ? ST_ZERO : (pv_col(pivot[l]) == int32_t(i) ? ST_OWNER : ST_ACTIVE);
        state[i] = st;
        if (rinfo && m > 0) {
            const int dm = rinfo[i];
            atomicMin(&smin[dm], c[0]);
            if (st == ST_ACTIVE) atomicMax(&smax[dm], l + 1);
        }
        if (app && st == ST_OWNER) {
            int4 v = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
            if (m <= 4) {
                v.x = int(m) - 1;
                if (m > 1) v.y = c[0];
                if (m > 2) v.z = c[1];
                if (m > 3) v.w = c[2];
            }
            app[l] = v;
        }
        nact += (st == ST_ACTIVE);
    }
    ncl = warp_sum(ncl);
    nact = warp_sum(nact);
    if ((threadIdx.x & 31) == 0) {
        if (ncl) cnt_add(&counters[CNT_CLEARED], ncl);
        if (nact) cnt_add(&counters[CNT_ACTIVE], nact);
    }
    if (rinfo) {
        __syncthreads();
        if (threadIdx.x < kNumDims) {
            if (smin[threadIdx.x] != INT_MAX) atomicMin(&info->min_row[threadIdx.x], smin[threadIdx.x]);
            if (smax[threadIdx.x] >= 0) atomicMax(&info->max_row[threadIdx.x], smax[threadIdx.x]);
        }
    }
}

// per-dimension min first row over non-empty columns and max low + 1 over
// active columns (ColumnShrink, include/specseq.h:374-398)
__global__ void k_dim_rows(int64_t n, const int32_t* rdim, const int32_t* arena, const uint64_t* desc,
                           const int32_t* low, const uint8_t* state, DimInfo* info) {
    __shared__ int smin[kNumDims], smax[kNumDims];
    if (threadIdx.x < kNumDims) { smin[threadIdx.x] = INT_MAX; smax[threadIdx.x] = -1; }
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint64_t d = desc[i];
        uint32_t len = desc_len(d);
        if (!len) continue;
        int dm = rdim[i];
        atomicMin(&smin[dm], arena[desc_off(d) + kHdr]);
        if (state[i] == ST_ACTIVE) atomicMax(&smax[dm], low[i] + 1);
    }
    __syncthreads();
    if (threadIdx.x < kNumDims) {
        if (smin[threadIdx.x] != INT_MAX) atomicMin(&info->min_row[threadIdx.x], smin[threadIdx.x]);
        if (smax[threadIdx.x] >= 0) atomicMax(&info->max_row[threadIdx.x], smax[threadIdx.x]);
    }
}

__global__ void k_diminfo_reset(DimInfo* info) {
    int d = threadIdx.x;
    if (d < kNumDims) { info->min_row[d] = INT_MAX; info->max_row[d] = -1; }
}

int init_passes(Device& D, bool lows_done, cudaStream_t s) {
    const int64_t n = D.n;
    const unsigned g = grid_for(n, 256) > 65536 ? 65536 : grid_for(n, 256);
    if (!lows_done) k_init_low<<<g, 256, 0, s>>>(n, D.arena, D.desc, D.low, D.leftmost);
    k_init_apparent<<<g, 256, 0, s>>>(n, D.arena, D.desc, D.low, D.leftmost, D.pivot, D.cleared, D.negative,
                                      D.counters);
    return lows_done ? 1 : 2;
}

int init_compress(Device& D, const uint8_t* dropped, bool keep_rows, bool final, cudaStream_t s, int64_t cb,
                  int64_t ce, bool reset) {
    const int64_t n = ce < 0 ? D.n : ce;
    if (n <= cb) return 0;
    // the row bounds go to the DimInfo through a few atomics per block: few blocks
    const unsigned g = grid_for(n - cb, 256) > 4096 ? 4096 : grid_for(n - cb, 256);
    if (final && reset) k_diminfo_reset<<<1, 32, 0, s>>>(D.diminfo);
    k_init_compress<<<g, 256, 0, s>>>(cb, n, D.arena, D.desc, D.low, D.pivot, D.cleared, D.negative, D.state, dropped,
                                      keep_rows, final ? D.app : nullptr, final ? D.dim : nullptr, D.diminfo,
                                      D.counters, D.err);
    return final && reset ? 2 : 1;
}

// Inline copies of the short apparent columns, by row (see Device::app).
__global__ void k_build_apparent(int64_t n, const uint64_t* pivot, const int32_t* arena, int4* app) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        int4 v = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
        const uint64_t e = pivot[r];
        if (e != kNoOwner) {
            const int32_t* h = arena + pv_slot(e);
            const int len = h[0];
            if (len >= 1 && len <= 4 && h[kHdr + len - 1] == int32_t(r)) {
                v.x = len - 1;
                if (len > 1) v.y = h[kHdr];
                if (len > 2) v.z = h[kHdr + 1];
                if (len > 3) v.w = h[kHdr + 2];
            }
        }
        app[r] = v;
    }
}

int build_apparent(Device& D, cudaStream_t s) {
    const int64_t n = D.n;
    if (n == 0) return 0;
    k_build_apparent<<<grid_for(n, 256) > 65536 ? 65536 : grid_for(n, 256), 256, 0, s>>>(n, D.pivot, D.arena, D.app);
    return 1;
}

// Active list in reordered order (dimension segments are contiguous) and the
// per-dimension bounds.
__global__ void k_act_segments(const int64_t* actpos, int64_t n, DimInfo* info) {
    int d = threadIdx.x;
    if (d < kNumDims) {
        int32_t b = info->col_begin[d], e = info->col_end[d];
        info->act_begin[d] = int32_t(b < n ? actpos[b] : actpos[n]);
        info->act_end[d] = int32_t(e < n ? actpos[e] : actpos[n]);
    }
}

int active_list(Device& D, bool rows_done, cudaStream_t s) {
    const int64_t n = D.n;
    const uint8_t* state = D.state;
    int32_t* act = D.active;
    int64_t* pos = D.scratch64;
    scan([=] __device__(int64_t i) -> int64_t { return state[i] == ST_ACTIVE ? 1 : 0; },
         [=] __device__(int64_t i, int64_t pre, int64_t v) {
             pos[i] = pre;
             if (v) act[pre] = int32_t(i);
         },
         n, D.blk, s);
    // pos[n] = total
    cudaMemcpyAsync(pos + n, D.blk + scan_blocks(n), sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
    k_act_segments<<<1, 32, 0, s>>>(pos, n, D.diminfo);
    if (rows_done) return 4;
    k_diminfo_reset<<<1, 32, 0, s>>>(D.diminfo);
    const unsigned g = grid_for(n, 256) > 4096 ? 4096 : grid_for(n, 256);
    k_dim_rows<<<g, 256, 0, s>>>(n, D.dim, D.arena, D.desc, D.low, D.state, D.diminfo);
    return 6;
}

// ------------------------------------------------------------------- pairs
// primal: row r (reordered) owned by column c -> (perm[r], perm[c]).
// dual: the dual row r' owned by dual column c' maps back to the primal pair
// (n-1-c', n-1-r') of the dualized matrix's own numbering; `dual_to_input`
// then maps those primal reordered indices to input indices.
__global__ void k_pairs_scatter(int64_t n, const uint64_t* pivot, const int32_t* perm, int64_t* death_of,
                                uint8_t* paired, int dual) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        uint64_t e = pivot[r];
        if (e == kNoOwner) continue;
        int32_t c = pv_col(e);
        int64_t birth, death;
        if (!dual) {
            birth = perm[r];
            death = perm[c];
        } else {
            birth = perm[n - 1 - c];
            death = perm[n - 1 - r];
        }
        death_of[birth] = death;
        paired[birth] = 1;
        paired[death] = 1;
    }
}

__global__ void k_mark_dropped(int64_t n, const uint8_t* dropped, const int32_t* perm, uint8_t* paired) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        if (dropped[i]) paired[perm[i]] = 1;
}

int extract_pairs(Device& D, int dual, const uint8_t* dropped, cudaStream_t s) {
    const int64_t n = D.n;
    const unsigned g = grid_for(n, 256) > 65536 ? 65536 : grid_for(n, 256);
    fill_i64(D.death_of, -1, n, s);
    cudaMemsetAsync(D.negative, 0, n, s);  // reused as the "paired or dropped" mark
    k_pairs_scatter<<<g, 256, 0, s>>>(n, D.pivot, D.perm, D.death_of, D.negative, dual);
    if (dropped) k_mark_dropped<<<g, 256, 0, s>>>(n, dropped, D.perm, D.negative);
    const int64_t* death_of = D.death_of;
    int64_t* pairs = D.pairs;
    scan([=] __device__(int64_t i) -> int64_t { return death_of[i] >= 0 ? 1 : 0; },
         [=] __device__(int64_t i, int64_t pre, int64_t v) {
             if (v) {
                 pairs[2 * pre] = i;
                 pairs[2 * pre + 1] = death_of[i];
             }
         },
         n, D.blk, s);
    cudaMemcpyAsync(&D.counters[CNT_NPAIRS], D.blk + scan_blocks(n), sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
    const uint8_t* paired = D.negative;
    int64_t* ess = D.ess;
    scan([=] __device__(int64_t i) -> int64_t { return paired[i] ? 0 : 1; },
         [=] __device__(int64_t i, int64_t pre, int64_t v) {
             if (v) ess[pre] = i;
         },
         n, D.blk, s);
    cudaMemcpyAsync(&D.counters[CNT_NESS], D.blk + scan_blocks(n), sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
    return 8 + (dropped ? 1 : 0);
}

}  // namespace sspp
