/*
 * sspp.h - C ABI of the B200 persistent-homology reduction engine.
 *
 * The reference (SpecSeq++) exposes no library API: its only entry points are
 * the `specseq++` command line (src/main.cu:269-352) and the header-only C++
 * class SpecSeqPlusPlus (include/specseq.h:63-1194).  Every function below
 * names the reference interface it replaces.  Conventions: plain pointers and
 * sizes, no CUDA or torch types; int status codes (SSPP_OK = 0) instead of the
 * reference's exit(EXIT_FAILURE) (include/kernel.h:26-32); the caller owns
 * input buffers, the context owns all device state; one context per host
 * thread.  Streams are passed as `void*` holding a cudaStream_t (NULL = the
 * context's own stream).
 */
#ifndef SSPP_H_
#define SSPP_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SSPP_OK 0
#define SSPP_ERR_BAD_INPUT 1  /* malformed matrix, bad parameter, bad file       */
#define SSPP_ERR_CAPACITY 2   /* device arena or a size limit exhausted          */
#define SSPP_ERR_CUDA 3       /* a CUDA runtime call failed                      */
#define SSPP_ERR_TIMEOUT 4    /* a bounded device loop hit its iteration limit   */
#define SSPP_ERR_STATE 5      /* call out of order (e.g. compute before init)    */
#define SSPP_ERR_IO 6         /* file could not be opened / written              */

/* file formats of src/main.cu:34-37 */
#define SSPP_ASCII 0
#define SSPP_BINARY 1

typedef struct sspp_ctx sspp_ctx;

typedef struct sspp_config {
    int32_t device;          /* CUDA device ordinal                                  */
    int64_t arena_bytes;     /* initial column arena; 0 = sized from the input       */
    int32_t verbose;         /* 0 = silent                                           */
    int32_t profile;         /* 1 = time every device phase with CUDA events         */
    int32_t host_threads;    /* host threads for staged copies; 0 = all cores         */
    int32_t sm_share;        /* persistent reduction launches use 1/sm_share of the
                                GPU (contexts that run side by side, e.g. a server's
                                workers); 0 or 1 = the whole GPU.  Above 1 the
                                autotuner also tries no candidate on inputs of 2^20
                                columns or more (a slow trial would delay the other
                                contexts' work)                                      */
} sspp_config;

/* The reference's 12 positional CLI values (src/main.cu:281-294) minus file
 * names/formats.  `autotune` = 1 replaces ss_block_size, growth, queue_size,
 * the level capacities and heavy_threads with the engine's choice for the
 * input's size class (a process-wide history of measured candidates; the
 * reference sets these by hand); 2 also lets it choose between dualize 0 and
 * 2, which never changes the pairs. */
typedef struct sspp_params {
    int32_t dualize;          /* 0 boundary matrix; 1 coboundary (anti-transpose) as
                                 the reference; 2 the 0-dimensional pairs from the
                                 boundary matrix's edges, then the coboundary matrix
                                 from dimension 1 up (no counterpart in the
                                 reference); the pairs are the same in every mode   */
    int32_t model;            /* bit0 high-dimension guided clearing, bit1 collapse   */
    int32_t max_iteration;    /* candidates per simplex for guided clearing           */
    int32_t ss_block_size;    /* initial spectral-sequence block size                 */
    float growth;             /* block_size_growth_rate (>= 1)                        */
    int32_t queue_size;       /* concurrent column workers per launch                 */
    int32_t level1_capacity;  /* per-worker on-chip column capacity (ints)            */
    int32_t level2_capacity;  /* per-block on-chip column capacity (ints)             */
    int32_t autotune;         /* 0 off, 1 launch parameters, 2 also dualization     */
    int32_t heavy_threads;    /* threads per heavy-tier column: 128 or 256 (0 = 256)  */
    int32_t representatives;  /* 1: keep whole reduced columns so that sspp_representative
                                 can return each pair's cycle (dualize 0 only; skips the
                                 negative-row compression, so the reduction does more work) */
    int32_t schedule;         /* how the spectral-sequence blocks are driven: 1 a host
                                 loop of per-block launches (as the reference's
                                 GPU_Compute); 2 one persistent launch draining a device
                                 queue of (complex, block) items, each complex with its
                                 own block order and dimension gate; 0 = 1.  The
                                 pairs are the same either way */
} sspp_params;

/* Per-run counters (device-side counters plus host timings). */
typedef struct sspp_stats {
    int64_t ncols, nnz;
    int64_t active_after_init;   /* columns left for the reduction after init     */
    int64_t apparent_pairs;      /* pivots found by the init pass                  */
    int64_t cleared_init;        /* columns cleared by the init pass               */
    int64_t highclear_cleared;   /* top-dimension columns cleared by guided clear  */
    int64_t collapse_dropped;    /* columns removed by edge collapse               */
    int64_t additions;           /* column additions performed on the device       */
    int64_t add_ints;            /* sum of |a| + |b| + |a xor b| over additions    */
    int64_t published_ints;      /* arena ints written by the reduction            */
    int64_t displaced;           /* pivot owners displaced by smaller columns      */
    int64_t ss_steps;            /* spectral-sequence launches                     */
    int64_t npairs, nessential;
    double init_ms, compute_ms;  /* GPU_Init / GPU_Compute equivalents            */
    int64_t launches;            /* kernels launched by the last init + compute    */
    /* device time per phase (profile = 1 only): init passes, light-tier and
     * heavy-tier reduction launches, pair extraction */
    double init_gpu_ms, light_gpu_ms, heavy_gpu_ms, pairs_gpu_ms;
    int64_t light_launches, heavy_launches;
    int64_t arena_ints_used;     /* column arena in use after the reduction (ints)  */
    int64_t tuned_candidate;     /* autotuner candidate of the last run, or -1     */
    int64_t heavy_additions;     /* additions done by the CTA tier                 */
    double build_ms;             /* last sspp_load_rips / sspp_load_lowerstar (host
                                    clock, input staging included), else 0          */
    int64_t heavy_fast_inline;   /* CTA-tier additions of short apparent addends    */
    int64_t heavy_fast_slot;     /* CTA-tier additions of short published addends   */
} sspp_stats;

/* Replaces: the SpecSeqPlusPlus constructor's allocation (include/specseq.h:486-512). */
sspp_ctx* sspp_create(const sspp_config* cfg);
void sspp_destroy(sspp_ctx* ctx);
const char* sspp_last_error(const sspp_ctx* ctx);
/* Fills *p with the reference's defaults (README.md:26-51): no dualize,
 * model 0, max_iteration 0, ss_block_size 102400, growth 1.05,
 * queue_size 65536, level capacities 1000 / 8000 (and schedule 0). */
void sspp_default_params(sspp_params* p);

/* Replaces: processFiles (src/main.cu:90-167).  fmt = SSPP_ASCII / SSPP_BINARY.
 * Ascii indices are 0-based face indices; binary is PHAT's int64 layout (the
 * reference skips the +1 shift for binary files, src/main.cu:146-155; here both
 * formats are read the same way). */
int32_t sspp_load_phat(sspp_ctx* ctx, const char* path, int32_t fmt);

/* Replaces: the hv_csc / hv_dim vectors handed to the SpecSeqPlusPlus
 * constructor (src/main.cu:324-335).  Host arrays in filtration order:
 * dims[ncols], col_ptr[ncols+1] (int64), rows[col_ptr[ncols]] with each column's
 * face indices ascending and unique.  Copied to the device at once. */
int32_t sspp_load_csc(sspp_ctx* ctx, int64_t ncols, const int32_t* dims, const int64_t* col_ptr, const int32_t* rows);

/* Same, for arrays already resident in device memory: nothing is copied, the
 * context reads them in place, so they must stay valid and unmodified until
 * the next load or sspp_destroy.  Validated on the device. */
int32_t sspp_load_csc_device(sspp_ctx* ctx, int64_t ncols, const int32_t* d_dims, const int64_t* d_col_ptr,
                             const int32_t* d_rows);

/* Builds on the device, and loads as the input matrix, the Vietoris-Rips
 * complex of npts points (npts x space_dim float32, row-major, space_dim 1..3,
 * in host memory or in device memory of the context's device): an edge joins
 * two points whose float32 Euclidean distance (coordinate differences squared
 * and summed in order, then the square root, each step rounded to nearest) is
 * <= radius; every clique of up to maxdim + 1 (<= 4) points is a simplex whose
 * value is its longest edge; vertices have value 0.  Columns are in (value,
 * dimension, lexicographic vertex tuple) order, faces ascending, as in the
 * reference's input files, which external tools write
 * (phat-highclear/addons/rips.cpp; read by src/main.cu:90-167).
 * Non-finite coordinates are BAD_INPUT. */
int32_t sspp_load_rips(sspp_ctx* ctx, int64_t npts, int32_t space_dim, const float* points, float radius,
                       int32_t maxdim);

/* Same, for the lower-star filtration of the Freudenthal (Kuhn) triangulation
 * of a gx x gy x gz grid: values[gx * gy * gz] (x fastest, then y, then z; host
 * or device memory) on the vertices, a simplex's value the largest of its
 * vertices'; vertex v + (dx, dy, dz) for every non-zero 0/1 offset is joined to
 * v.  -0 is read as +0; NaN is BAD_INPUT.  Every simplex up to maxdim (<= 3). */
int32_t sspp_load_lowerstar(sspp_ctx* ctx, int64_t gx, int64_t gy, int64_t gz, const float* values,
                            int32_t maxdim);

/* A complex to build on the device: a point cloud's Vietoris-Rips complex
 * (kind SSPP_BUILD_RIPS: size[0] points of size[1] coordinates in `data`,
 * `radius`) or a grid field's lower-star filtration (SSPP_BUILD_LOWERSTAR:
 * size[0] x size[1] x size[2] values in `data`), each as sspp_load_rips /
 * sspp_load_lowerstar describe; `data` in host memory or in device memory of
 * the context's device. */
#define SSPP_BUILD_RIPS 0
#define SSPP_BUILD_LOWERSTAR 1
typedef struct sspp_build_spec {
    int32_t kind;
    int32_t maxdim;
    int64_t size[3];
    const float* data;
    float radius;
} sspp_build_spec;

/* Builds k complexes on the device, one after another, and loads them as one
 * batch (as sspp_load_batch_device: block-diagonal, results per complex in
 * its own indices).  No counterpart in the reference, which reads one file per
 * process.  sspp_batch_values copies complex i's column filtration values and
 * returns its column count (-1 on error). */
int32_t sspp_load_built_batch(sspp_ctx* ctx, int32_t k, const sspp_build_spec* specs);
int64_t sspp_batch_values(sspp_ctx* ctx, int32_t i, float* out, int64_t cap);

/* The matrix the context reduces (after any load; a batch's is the block-
 * diagonal concatenation) and, after sspp_load_rips / sspp_load_lowerstar,
 * each column's filtration value.  Any output may be NULL; asking for values
 * of a matrix that was not built is BAD_INPUT. */
int32_t sspp_input_size(sspp_ctx* ctx, int64_t* ncols, int64_t* nnz);
int32_t sspp_input_copy(sspp_ctx* ctx, int32_t* dims, int64_t* col_ptr, int32_t* rows, float* values);

/* Replaces: SpecSeqPlusPlus::GPU_Init (include/specseq.h:513-590): dimension
 * reorder, edge collapse, guided clearing, init passes, dualization, active
 * lists.  Blocks until done. */
int32_t sspp_init(sspp_ctx* ctx, const sspp_params* p, void* stream);

/* Replaces: SpecSeqPlusPlus::GPU_Compute (include/specseq.h:592-1060): the
 * spectral-sequence reduction, entirely on the device (no CPU tail stage).
 * Blocks until done. */
int32_t sspp_compute(sspp_ctx* ctx, void* stream);

/* sspp_init + sspp_compute. */
int32_t sspp_reduce(sspp_ctx* ctx, const sspp_params* p, void* stream);

/* Replaces: GetPersistencePairs (include/specseq.h:1182-1193).  Pairs in input
 * (0-based) indices, sorted by (birth, death), written as birth,death int64
 * pairs.  Returns the number of pairs, or -1 on error; copies at most cap pairs. */
int64_t sspp_num_pairs(sspp_ctx* ctx);
int64_t sspp_pairs(sspp_ctx* ctx, int64_t* out_birth_death, int64_t cap);

/* Essential (never paired) simplices in input indices, ascending; simplices
 * removed by edge collapse are not listed.  The reference does not report
 * these; PHAT's pair files do not either. */
int64_t sspp_num_essential(sspp_ctx* ctx);
int64_t sspp_essentials(sspp_ctx* ctx, int64_t* out, int64_t cap);

/* Batching (no counterpart in the reference, which reduces one file per
 * process).  k independent complexes, each with its own 0-based face indices,
 * are loaded as one block-diagonal matrix: columns of different complexes
 * never share rows, so one reduction yields every complex's pairs and all
 * kernels drain the columns of all complexes from the same work counters.
 * sspp_load_batch takes host arrays per complex; sspp_load_batch_device takes
 * one device-resident concatenation whose face indices are already offset by
 * the columns of the complexes before them.  After sspp_reduce, per-complex
 * results come back in the complex's own indices. */
int32_t sspp_load_batch(sspp_ctx* ctx, int32_t k, const int64_t* ncols, const int32_t* const* dims,
                        const int64_t* const* col_ptr, const int32_t* const* rows);
int32_t sspp_load_batch_device(sspp_ctx* ctx, int32_t k, const int64_t* ncols, const int32_t* d_dims,
                               const int64_t* d_col_ptr, const int32_t* d_rows);
int64_t sspp_batch_num_pairs(sspp_ctx* ctx, int32_t i);
int64_t sspp_batch_pairs(sspp_ctx* ctx, int32_t i, int64_t* out_birth_death, int64_t cap);
int64_t sspp_batch_num_essential(sspp_ctx* ctx, int32_t i);
int64_t sspp_batch_essentials(sspp_ctx* ctx, int32_t i, int64_t* out, int64_t cap);
/* Bulk form for large batches: sspp_batch_counts writes every complex's pair
 * and essential counts (arrays of k, either may be NULL); sspp_batch_copy then
 * fills pairs_out[i] (2 * npairs[i] int64) and ess_out[i] (ness[i] int64) in
 * the complexes' own indices in one staged copy (NULL entries are skipped). */
int32_t sspp_batch_counts(sspp_ctx* ctx, int64_t* npairs, int64_t* ness);
int32_t sspp_batch_copy(sspp_ctx* ctx, int64_t* const* pairs_out, int64_t* const* ess_out);

/* Host-side PHAT files, no device needed.  sspp_phat_read parses a boundary
 * matrix as processFiles does (src/main.cu:90-167; 0-based indices, every
 * column sorted and de-duplicated) on several host threads for large files;
 * the handle hands out its size and a copy of the arrays.  sspp_phat_write
 * writes a matrix in either format (the layout sspp_phat_read accepts). */
typedef struct sspp_phat sspp_phat;
sspp_phat* sspp_phat_read(const char* path, int32_t fmt, char* err_msg, int32_t err_cap);
int64_t sspp_phat_ncols(const sspp_phat* h);
int64_t sspp_phat_nnz(const sspp_phat* h);
int32_t sspp_phat_copy(const sspp_phat* h, int32_t* dims, int64_t* col_ptr, int32_t* rows);
void sspp_phat_free(sspp_phat* h);
int32_t sspp_phat_write(const char* path, int32_t fmt, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                        const int32_t* rows, char* err_msg, int32_t err_cap);

/* Replaces: the HIGHOUT build's out_maxdimclear (include/specseq.h:1108-1129,
 * Makefile:33-34).  Writes the loaded matrix, in input order and indices, with
 * the columns that guided clearing (model bit 1) clears and that the edge
 * collapse (model bit 2) drops written as dimension-only lines; every other
 * column as loaded.  Reducing the written file gives the same pairs.  The
 * guided clearing here walks the neighbour lists in the intended direction,
 * while the reference's walk only ever accepts the smallest common neighbour
 * (include/kernel.h:217), so more columns can be cleared than in the
 * reference's files.  Leaves the context loaded but not initialised (call
 * sspp_init again). */
int32_t sspp_export_preprocessed(sspp_ctx* ctx, const sspp_params* p, const char* path, int32_t fmt);

/* Replaces: writeVectorToFile (src/main.cu:191-229). */
int32_t sspp_write_pairs(sspp_ctx* ctx, const char* path, int32_t fmt);

/* No counterpart in the reference (PHAT's python binding returns pairs only).
 * A representative cycle of the pair whose death is `death` (an input index),
 * after a reduction with representatives = 1 and dualize = 0: the simplices of
 * the death column's reduced column, as input indices, ascending.  Over Z2 it
 * is the boundary of a chain whose youngest simplex is `death`, so it is a
 * cycle, and its youngest simplex is the pair's birth.  With edge collapse it
 * lies in the collapsed complex.  Copies up to cap entries to out and returns
 * the cycle's length, or -1 (sspp_last_error) when `death` kills no class, the
 * reduction kept no representatives, or the context holds a batch. */
int64_t sspp_representative(sspp_ctx* ctx, int64_t death, int64_t* out, int64_t cap);

int32_t sspp_get_stats(const sspp_ctx* ctx, sspp_stats* out);
/* The parameters the last sspp_init ran with (autotuned values included). */
int32_t sspp_get_params(const sspp_ctx* ctx, sspp_params* out);

/* Serving (no counterpart in the reference, whose CLI reduces one file per
 * process).  A resident request loop on one GPU: `workers` host threads, each
 * with its own context and stream, take the requests waiting in arrival order
 * as one batch (block-diagonal, as sspp_load_batch) as long as the batch's
 * device-memory estimate fits the worker's share of `memory_budget`; requests
 * that arrive while batches run join the next batch a worker forms, and the
 * workers' batches overlap on the device (copies of one with the reduction of
 * another).  Estimate per request: 128 bytes per column + 4 per entry + the
 * column arena, 4 bytes x fill x (nnz + 7 ncols), with fill the largest arena
 * fill the autotuner has seen for the request's size class (3 before any).
 * A request whose estimate exceeds the whole budget is refused at submit.
 * A batch that fails is re-run request by request so one bad input fails
 * alone.  Latency = completion - submission, on the host's steady clock. */
typedef struct sspp_server sspp_server;

typedef struct sspp_server_config {
    int32_t device;
    int32_t workers;             /* concurrent batches (contexts, streams); 0 = 2   */
    int64_t memory_budget;       /* bytes for all workers; 0 = 85% of free memory   */
    int64_t max_batch_cols;      /* 0 = no limit besides memory                     */
    int32_t max_batch_requests;  /* 0 = no limit                                    */
    double batch_window_ms;      /* wait this long for more requests when the queue
                                    holds fewer than max_batch_requests; 0 = none   */
} sspp_server_config;

typedef struct sspp_server_stats {
    int64_t submitted, completed, failed, rejected, batches, columns;
    double wall_s;               /* first submission to last completion            */
    double cols_per_s;           /* columns of completed requests / wall_s         */
    double p50_ms, p95_ms, p99_ms, max_ms, mean_ms;
    double mean_batch_requests;
    double load_s, reduce_s, results_s;  /* host time in each batch phase, summed
                                            over workers                        */
} sspp_server_stats;

/* request states */
#define SSPP_REQ_QUEUED 0
#define SSPP_REQ_RUNNING 1
#define SSPP_REQ_DONE 2
#define SSPP_REQ_FAILED 3

/* submit flag: the caller keeps dims / col_ptr / rows valid and unmodified
 * until the request is done (no copy at submission) */
#define SSPP_SUBMIT_NOCOPY 1
/* submit flag (point clouds and fields): keep the built matrix's filtration
 * values for sspp_server_values */
#define SSPP_SUBMIT_VALUES 2

/* params: as for sspp_init (autotune applies per batch). */
sspp_server* sspp_server_create(const sspp_server_config* cfg, const sspp_params* params);
/* Finishes every accepted request, then stops the workers. */
void sspp_server_destroy(sspp_server* srv);
const char* sspp_server_last_error(sspp_server* srv);
/* Returns the request id (>= 0), or -SSPP_ERR_* when refused. */
int64_t sspp_server_submit(sspp_server* srv, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                           const int32_t* rows, int32_t flags);
/* A request given as a point cloud or a scalar field (as sspp_load_rips /
 * sspp_load_lowerstar): a worker builds the point-cloud and field requests it
 * takes together on the device, one after another, and reduces them as one
 * block-diagonal batch (sspp_load_built_batch; matrices and built requests are
 * never mixed in a batch); a request's pairs and essentials are
 * indices of its built matrix, whose column values sspp_server_values returns
 * when submitted with SSPP_SUBMIT_VALUES.  A field's request is admitted by an
 * upper bound of its size (26 columns and 74 entries per vertex); a point
 * cloud's size is known only once built, and one that does not fit the
 * device fails with SSPP_ERR_CAPACITY.  The reference builds such complexes
 * with external tools (phat-highclear/addons/rips.cpp) and serves nothing. */
int64_t sspp_server_submit_rips(sspp_server* srv, int64_t npts, int32_t space_dim, const float* points, float radius,
                                int32_t maxdim, int32_t flags);
int64_t sspp_server_submit_lowerstar(sspp_server* srv, int64_t gx, int64_t gy, int64_t gz, const float* values,
                                     int32_t maxdim, int32_t flags);
/* Copies up to cap values and returns the built matrix's column count, or -1. */
int64_t sspp_server_values(sspp_server* srv, int64_t id, float* out, int64_t cap);
/* SSPP_OK once the request is done or failed, SSPP_ERR_TIMEOUT if timeout_ms
 * passed first (timeout_ms < 0 waits for ever), SSPP_ERR_STATE for an unknown id. */
int32_t sspp_server_wait(sspp_server* srv, int64_t id, double timeout_ms);
/* SSPP_REQ_* state, or -SSPP_ERR_STATE for an unknown id. */
int32_t sspp_server_state(sspp_server* srv, int64_t id);
/* Status code of a finished request (SSPP_OK or the failure); its message. */
int32_t sspp_server_result(sspp_server* srv, int64_t id, char* msg, int32_t msg_cap);
int64_t sspp_server_num_pairs(sspp_server* srv, int64_t id);
int64_t sspp_server_pairs(sspp_server* srv, int64_t id, int64_t* out_birth_death, int64_t cap);
int64_t sspp_server_num_essential(sspp_server* srv, int64_t id);
int64_t sspp_server_essentials(sspp_server* srv, int64_t id, int64_t* out, int64_t cap);
/* Latency of a finished request (ms), -1 otherwise. */
double sspp_server_latency_ms(sspp_server* srv, int64_t id);
/* Frees a finished request's results and forgets the id. */
int32_t sspp_server_release(sspp_server* srv, int64_t id);
int32_t sspp_server_get_stats(sspp_server* srv, sspp_server_stats* out);
/* Clears the latency record and counters (not the autotuner history). */
int32_t sspp_server_reset_stats(sspp_server* srv);

/* No counterpart in the reference.  Allocation-free reduction for callers that
 * cannot have a library allocate device memory (a server that reserves all of
 * its GPU memory up front; a multi-stream pipeline that cannot afford the
 * device-wide synchronisation of cudaMalloc/cudaFree).  All working memory is
 * one 64 MiB file-scope device array that every GPU loading this library holds
 * until exit.  Inputs (filtration order, as sspp_load_csc) and outputs are
 * device pointers: d_pairs receives up to ncols (birth, death) int64 pairs
 * sorted by birth (room for 2 * ncols int64), *d_npairs their number.  Limits:
 * ncols <= 1048576 and 3 * ncols + nnz <= 12582896, else SSPP_ERR_BAD_INPUT;
 * fill-in beyond the array gives SSPP_ERR_CAPACITY; a col_ptr that does not
 * run from 0 to nnz without decreasing, a dimension outside 0..7, or faces that
 * are unsorted, out of range or not one dimension lower give
 * SSPP_ERR_BAD_INPUT.  The first call on a device looks up the array's address
 * (make it before any stream capture); calls that overlap on the GPU share the
 * array and race, so serialise them.  Each call copies the status word back and
 * synchronises the stream, so it returns once the reduction has finished; a
 * message is written to err_msg (may be NULL) when it fails. */
int32_t sspp_reduce_noalloc(int64_t ncols, int64_t nnz, const int32_t* d_dims, const int64_t* d_col_ptr,
                            const int32_t* d_rows, int64_t* d_pairs, int64_t* d_npairs, void* stream, char* err_msg,
                            int32_t err_cap);

#ifdef __cplusplus
}
#endif

#endif /* SSPP_H_ */
