/*
 * mr.h — C-ABI of the B200-native reordered-SpMV library (libmr.so).
 *
 * Drop-in boundary for the reordered-SpMV path of Zhangq388/MATRIX-REORDER.
 * Each entry point names the reference interface it replaces as
 * `file:line` in that project. The reference has no FFI layer of its own; its
 * operator API is the C++ template struct GRAPH<V> (include/class.cuh:58-97)
 * and the TILE / merbit_kernel templates (include/merbit.cuh). These entry
 * points are what a binding of that API binds.
 *
 * Conventions
 *  - Every call returns an mr_status (0 = MR_OK); no C++ exception crosses
 *    the ABI. mr_status_string() gives a message.
 *  - Matrices are textbook CSR: row i holds colidx[rowptr[i] .. rowptr[i+1]).
 *    (The reference stores the transpose: its `col_ind` is our row and its
 *    `row_ind` our column, src/class.cu:1342, :1372.)
 *  - Pointers named *_dev are device memory, *_host host memory. Matrix and
 *    vector buffers are owned by the caller; plan objects own their
 *    descriptors. Work is enqueued on `stream` (a cudaStream_t, NULL = the
 *    legacy default stream) and is ordered on it. Calls on different streams
 *    may run concurrently.
 *  - 32-bit indices: n_rows, n_cols and nnz must be < 2^31.
 */
#ifndef MR_H
#define MR_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mr_status {
    MR_OK = 0,
    MR_ERR_INVALID_ARG = 1,   /* bad size, null pointer or option */
    MR_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    MR_ERR_NOMEM = 3,         /* device or host allocation failed */
    MR_ERR_INVALID_PERM = 4,  /* permutation is not a bijection of [0, n) */
    MR_ERR_UNSUPPORTED = 5,   /* dtype / option not supported by this entry */
    MR_ERR_TIMEOUT = 6,       /* a bounded wait expired */
    MR_ERR_BUSY = 7,          /* admission refused: no slot / no memory */
    MR_ERR_NOT_FOUND = 8,     /* unknown id */
    MR_ERR_INTERNAL = 9,      /* a device-side consistency check failed */
    MR_ERR_PREDICT = 10       /* predictor produced a non-finite or <= 0 value */
} mr_status;

typedef enum mr_dtype {
    MR_F32 = 0,
    MR_F16 = 1,
    MR_BF16 = 2
} mr_dtype;

/* A CSR matrix in device memory (values of `dtype`). */
typedef struct mr_csr_view {
    int32_t n_rows;
    int32_t n_cols;
    int64_t nnz;
    const int32_t* rowptr; /* n_rows + 1 */
    const int32_t* colidx; /* nnz, sorted within each row for MERBIT/RD */
    const void* vals;      /* nnz */
    int32_t dtype;         /* mr_dtype */
} mr_csr_view;

const char* mr_status_string(int status);
int mr_version(void);
/* Last CUDA error text seen by this thread (empty if none). */
const char* mr_last_error(void);
/* Temporaries of every entry point come from a per-device stream-ordered
 * pool that keeps freed memory for the next call (no reference
 * counterpart). This returns the pool's unused memory of the current device
 * to the system; later calls grow it again. */
int mr_release_scratch(void);

/* *valid_host = 1 if rowptr[0] == 0, rowptr is non-decreasing,
 * rowptr[n_rows] == nnz and every column index is in [0, n_cols).
 * The SpMV entry points do not re-check this on every call; plan creation
 * and mr_permute_csr do. Synchronises `stream`. No reference counterpart
 * (the reference performs no input validation). */
int mr_csr_validate(const mr_csr_view* A, int* valid_host, void* stream);

/* ------------------------------------------------------------- SpMV ---- */

/* y = A x, FP32 x/y, values of A->dtype, FP32 accumulation. Plain CSR path.
 * Replaces the cusparseSpMV(CSR_ALG1) loop of GRAPH::spmv(env, "csr")
 * (src/class.cu:1359-1397). */
int mr_spmv_csr(const mr_csr_view* A, const float* x_dev, float* y_dev, void* stream);

/* MERBIT merge-path plan. The descriptor arrays are bit-identical to those
 * TILE<BLOCK,SIGMA>::TILE builds (include/merbit.cuh:134-155, Tile_Kernel
 * :55-131): tile_x/tile_y[tile_num+1] (bit 31 of tile_y = single-row tile)
 * and lane_desc[lane_num] (32-bit words for sigma < 15, 64-bit otherwise).
 * sigma: merge items per lane, 1..42 (reference 14; the SpMV kernels are
 * built for 7, 10, 14, 16, 20, 24, 28, 32). block: threads per CTA of the
 * SpMV kernel, 128, 256, 512 or 1024 (reference 256); 0 picks 1024. The
 * plan also owns the per-tile carry-out scratch.
 * The rowptr of A must stay unchanged while the plan is used. */
typedef struct mr_merbit_plan mr_merbit_plan;

typedef struct mr_merbit_plan_info {
    int32_t sigma;
    int32_t block;
    int32_t n_rows;
    int64_t nnz;
    int32_t lane_num;
    int32_t tile_num;
    int32_t desc_bytes;           /* 4 or 8 */
    const uint32_t* tile_x_dev;   /* tile_num + 1 */
    const uint32_t* tile_y_dev;   /* tile_num + 1 */
    const void* lane_desc_dev;    /* lane_num words of desc_bytes */
    int32_t hub_columns;          /* columns staged in shared memory (0: no hub cache) */
    double hub_coverage;          /* share of nonzeros whose x comes from the hub cache */
} mr_merbit_plan_info;

/* block 1024 (the default) selects the persistent kernel: one CTA of 32
 * warps per SM sweeping a contiguous range of tiles (ranges cut at plan
 * time by estimated cost), with the carry fix-up fused in. Its plan also
 * builds a hub cache when it pays: the most-used columns (as many as fit in
 * shared memory beside the staging buffers, and only if they take >= 20% of
 * the nonzeros) are staged in shared memory at
 * kernel start, and the plan keeps a copy of colidx with those columns
 * remapped — so such a plan snapshots the column indices of A, and must be
 * rebuilt if they change. block 128/256/512 select the tile-per-warp grid
 * kernel with a separate fix-up kernel. Results are bit-identical across
 * all forms. SpMVs that share one plan must not overlap on the GPU (the
 * plan owns the carry scratch). */
int mr_merbit_plan_create(const mr_csr_view* A, int sigma, int block, void* stream, mr_merbit_plan** plan);
#define MR_PLAN_NO_HUB_CACHE 1    /* never build the shared-memory hub cache */
#define MR_PLAN_GATHER_NO_L1 2    /* x gathers do not allocate L1 lines */
#define MR_PLAN_GATHER_L2_ONLY 4  /* x gathers read through L2 only (.cg) */
#define MR_PLAN_SMALL_HUB_CACHE 8 /* at most 8192 hub columns (leaves L1 room) */
#define MR_PLAN_HUB_LIMIT(kcols) ((int)(kcols) << 8) /* at most kcols * 1024 hub columns */
/* As mr_merbit_plan_create, with tuning flags (MR_PLAN_*); every flag
 * combination computes the same bits. */
int mr_merbit_plan_create_ex(const mr_csr_view* A, int sigma, int block, int flags, void* stream,
                             mr_merbit_plan** plan);
/* Replaces TILE::~TILE (include/merbit.cuh:256-263). Synchronises the device
 * before freeing. */
int mr_merbit_plan_destroy(mr_merbit_plan* plan);
int mr_merbit_plan_get_info(const mr_merbit_plan* plan, mr_merbit_plan_info* info);

/* y = A x with the MERBIT plan. Replaces the merbit_kernel<V,256,14> launch
 * loop of GRAPH::spmv(env, "merbit") (src/class.cu:1407-1430,
 * include/merbit.cuh:408-493). Deterministic: rows spanning tiles are
 * finished by an FP64 carry fix-up instead of float atomics, so no second
 * output buffer (the reference's d_z) is needed. A call uses the plan's
 * carry slots and completion counters: calls with the same plan must not
 * overlap on the GPU (order them on one stream or with events); calls with
 * different plans may. */
int mr_spmv_merbit(const mr_merbit_plan* plan, const mr_csr_view* A, const float* x_dev, float* y_dev, void* stream);

/* Allocation-free MERBIT SpMV: y = A x with no device allocation at all.
 * No counterpart in the reference (which allocates its plan and buffers
 * with cudaMalloc, include/merbit.cuh:146-151); it exists for callers that
 * cannot call cudaMalloc while they run SpMV, e.g. code whose device memory
 * is owned by another runtime's pool, or that must not synchronise the
 * device by allocating. The plan (SIGMA 14), carries and completion ticket
 * live in one file-scope device array sized for n_rows + nnz <= 2^24 merge
 * items (about 5.3 MB that every GPU which loads the library keeps until
 * exit); larger matrices return MR_ERR_UNSUPPORTED. The caller passes A, x
 * and y as for mr_spmv_merbit. Each call checks the matrix as plan creation
 * does and waits for that check on `stream` (a malformed rowptr or column
 * index returns MR_ERR_INVALID_ARG before any gather), then rebuilds the
 * plan into the array and gives bitwise the result of a planned call.
 * The first call on a device does a set-up: it looks up the array's device
 * address and keeps it, so make that first call before any stream capture
 * and make no call after cudaDeviceReset. All calls share the array, so
 * calls that overlap on the GPU race: order them on one stream. */
int mr_spmv_merbit_noalloc(const mr_csr_view* A, const float* x_dev, float* y_dev, void* stream);

/* ------------------------------------------------ batched SpMV ---- */

/* Many independent y_i = A_i x_i in one persistent launch per (sigma,
 * dtype) group, optionally replayed as a CUDA graph. No reference
 * counterpart: the reference runs one matrix per process; this is the
 * batched form of merbit_kernel (include/merbit.cuh:408-493). Each item's
 * result is bitwise identical to mr_spmv_merbit on that item alone. */
typedef struct mr_batch mr_batch;
typedef struct mr_batch_item {
    const mr_merbit_plan* plan;  /* plan of A (one plan may serve several items) */
    mr_csr_view A;               /* the matrix the plan was built for */
    const float* x;              /* device */
    float* y;                    /* device */
} mr_batch_item;

int mr_batch_create(const mr_batch_item* items, int32_t count, void* stream, mr_batch** batch);
int mr_batch_run(mr_batch* batch, void* stream);
/* Captures mr_batch_run into a CUDA graph owned by the batch (stream must
 * not be the legacy default stream); mr_batch_launch then replays it. */
int mr_batch_capture(mr_batch* batch, void* stream);
int mr_batch_launch(mr_batch* batch, void* stream);
/* Points item i at new x / y; a captured graph stays valid. Synchronises
 * `stream`. */
int mr_batch_set_vectors(mr_batch* batch, int32_t i, const float* x, float* y, void* stream);
int mr_batch_info(const mr_batch* batch, int32_t* groups, int64_t* total_tiles);
int mr_batch_destroy(mr_batch* batch);

/* Autotuner over MERBIT's tile size (sigma: items per lane, the tile is
 * 32 x sigma merge items), threads per CTA (block) and the hub cache: times
 * every supported combination on A (median of reps) and returns the fastest
 * as (sigma, block, plan flags for mr_merbit_plan_create_ex). The reference
 * hard-codes BLOCK 256, SIGMA 14 (src/class.cu:1409-1410). */
int mr_autotune_merbit(const mr_csr_view* A, const float* x_dev, float* y_dev, int32_t reps, int32_t* best_sigma,
                       int32_t* best_block, int32_t* best_flags, float* best_ms, void* stream);
/* Size-bucketed cache of tuning results: bucket = (floor(log2 rows),
 * floor(log2 mean row length)); a miss tunes on the given matrix. */
typedef struct mr_tuner mr_tuner;
int mr_tuner_create(mr_tuner** tuner);
int mr_tuner_destroy(mr_tuner* tuner);
int mr_tuner_pick(mr_tuner* tuner, const mr_csr_view* A, const float* x_dev, float* y_dev, int32_t* sigma,
                  int32_t* block, int32_t* flags, void* stream);
int mr_tuner_stats(mr_tuner* tuner, int32_t* buckets, int32_t* tuned);

/* ------------------------------------------------------- serving ---- */

/* Continuous-batching SpMV server over a device-resident pool of matrices.
 * No reference counterpart (the reference runs one matrix per process);
 * this is the serving form of the path. Matrices are registered with host
 * CSR arrays that the caller keeps alive, optionally with the permutation
 * perm[old] = new the matrix was reordered with; requests then carry x in
 * the original numbering and receive y in it. A matrix is uploaded and
 * planned on first use, within hbm_budget_bytes, evicting the least
 * recently used idle matrices. A scheduler thread batches the requests that
 * arrive within window_us of the first pending one (at most max_batch) and
 * keeps up to `lanes` batches in flight, pipelined (copies in, kernels,
 * copies out, each stage in launch order on its own stream). Each request's
 * result is bitwise the same alone or in any batch. */
typedef struct mr_server mr_server;
typedef struct mr_server_config {
    int64_t hbm_budget_bytes; /* device bytes for resident matrices; 0 = half the free memory */
    int32_t window_us;        /* batching window (default 200) */
    int32_t max_batch;        /* requests per batch (default 64) */
    int32_t lanes;            /* batches in flight, one buffer set each (default 3) */
    int32_t sigma;            /* MERBIT sigma of resident plans (default 14) */
    int32_t hub_cache;        /* nonzero: each resident matrix gets the single-matrix persistent plan
                                 (1024 threads, hub cache; about 4 more bytes of HBM per nonzero) and
                                 runs in its own launch instead of the batched kernel (default 0) */
} mr_server_config;
typedef struct mr_server_stats {
    int64_t submitted, completed, rejected, batches, admissions, evictions;
    int64_t resident_bytes, resident_matrices;
    double mean_batch;
    double p50_us, p99_us, mean_us, max_us; /* latency: submit -> result in y */
    double req_per_s;                       /* completed / (last completion - first submit) */
    /* per-stage time summed over batches (ms): device time of each batch's
     * H2D copies (from its first copy, waiting included), its kernels, its
     * D2H copies; host time the scheduler spent issuing batches */
    double h2d_ms, compute_ms, d2h_ms, launch_ms;
} mr_server_stats;

int mr_server_create(const mr_server_config* cfg, mr_server** server);
int mr_server_add_matrix(mr_server* server, int32_t n, int64_t nnz, const int32_t* rowptr_host,
                         const int32_t* colidx_host, const void* vals_host, int32_t dtype,
                         const int32_t* perm_old2new_host, int32_t* id);
/* Queues y = A_id x; x_host must stay valid and y_host writable until the
 * request completes (mr_server_wait / mr_server_drain). Vectors in
 * page-locked host memory (cudaHostAlloc, or cudaHostRegister covering the
 * whole vector) are copied by DMA straight from / into the caller's buffer;
 * other host memory is staged through the server's pinned buffers. Whether
 * an address is page-locked is looked up once per server (a buffer that
 * changes kind at the same address is still copied correctly). */
int mr_server_submit(mr_server* server, int32_t id, const float* x_host, float* y_host, uint64_t* ticket);
/* Waits up to timeout_ms (MR_ERR_TIMEOUT after); returns the request's status. */
int mr_server_wait(mr_server* server, uint64_t ticket, int32_t timeout_ms, double* latency_us);
int mr_server_drain(mr_server* server, int32_t timeout_ms);
int mr_server_get_stats(mr_server* server, mr_server_stats* stats);
int mr_server_reset_stats(mr_server* server);
int mr_server_destroy(mr_server* server);
/* Open-loop Poisson load generator: n_requests arrivals at `rate` per second
 * over the ids (uniform), x_of[k] / y_of[k] host buffers of ids[k]. */
int mr_server_loadgen(mr_server* server, const int32_t* ids, int32_t n_ids, int64_t n_requests, double rate,
                      uint64_t seed, const float* const* x_of, float* const* y_of, int32_t timeout_ms);

/* The plain per-request path the server is compared with: request r runs
 * alone on `stream` (H2D x, x' = P x, MERBIT SpMV with plans[req_mat[r]],
 * y = P^T y', D2H, synchronise). views/plans/perm_dev per matrix; x_host /
 * y_host per request, page-locked ones copied directly as in
 * mr_server_submit; elapsed_ms and lat_us (per request) may be NULL. */
int mr_plain_requests(int32_t n_mats, const mr_merbit_plan* const* plans, const mr_csr_view* views,
                      const int32_t* const* perm_dev, int64_t n_requests, const int32_t* req_mat,
                      const float* const* x_host, float* const* y_host, void* stream, double* elapsed_ms,
                      double* lat_us);

/* Gather ceiling of a column-index stream: time per pass (ms, mean of reps
 * after two warm-up passes) of a kernel that streams colidx / vals with
 * 16-byte evict-first loads and gathers x[colidx[k]] once per nonzero, with
 * no row structure and no y. A lower bound for any SpMV that gathers x once
 * per nonzero on the same stream; no reference counterpart (measurement
 * only). colidx and vals 16-byte aligned; the last nnz % 4 entries are left
 * out. */
int mr_gather_ceiling(const int32_t* colidx_dev, const float* vals_dev, int64_t nnz, const float* x_dev,
                      int32_t reps, float* ms_per_pass, void* stream);

/* ------------------------------------------------------ permutation ---- */

/* B = P A P^T: B[perm[r], perm[c]] = A[r, c], columns sorted within rows,
 * equal columns kept in source order. Output arrays are caller-allocated
 * (n_rows+1, nnz, nnz of A->dtype); the matrix must be square.
 * Replaces the perm scatter + gather relabel + GRAPH::sort(false) + coo2csr
 * of GRAPH::gorder4 (src/class.cu:2686-2705, :423-457, :1342).
 * Synchronises `stream` and returns MR_ERR_INVALID_PERM if perm is not a
 * bijection (output then undefined). */
int mr_permute_csr(const mr_csr_view* A, const int32_t* perm_old2new_dev,
                   int32_t* out_rowptr_dev, int32_t* out_colidx_dev, void* out_vals_dev, void* stream);

/* out[perm[i]] = in[i] when inverse == 0 (x' = P x), out[i] = in[perm[i]]
 * when inverse != 0 (y = P^T y', the check gather of src/class.cu:1437-1440). */
int mr_permute_vector(int32_t n, const int32_t* perm_old2new_dev, const float* in_dev, float* out_dev,
                      int inverse, void* stream);

/* perm_new2old[perm_old2new[i]] = i (the scatter of src/class.cu:2688-2689). */
int mr_perm_invert(int32_t n, const int32_t* perm_dev, int32_t* inv_dev, void* stream);

/* *valid_host = 1 if perm is a bijection of [0, n). Replaces check_perm
 * (include/utils.cuh:5-55), which only prints. Synchronises `stream`. */
int mr_check_perm(const int32_t* perm_dev, int32_t n, int* valid_host, void* stream);

/* ------------------------------------------- reuse-distance features ---- */

/* Exact sector reuse-distance histogram of the x-access stream (colidx in
 * CSR order): sector = col / sector_size; for each reuse, RD = number of
 * distinct sectors touched since the previous use; counts[b] for
 * b = upper_bound(edges, RD). counts_host has nedges+1 entries; *valid_host
 * gets the number of reuses. Counts are exact (integers). Replaces
 * compute_sector_rd_histogram (src/class.cu:892-936), whose probabilities are
 * counts[b] / valid. Synchronises `stream`. */
int mr_rd_hist_exact(const int32_t* stream_dev, int64_t nnz, int32_t ncols, int32_t sector_size,
                     const int32_t* edges_host, int32_t nedges, int64_t* counts_host, int64_t* valid_host,
                     void* stream);

/* Sampled reuse distance with HyperLogLog registers, same samples, statuses
 * and estimates as sampled_hll_rd_block_gpu (src/class.cu:1133-1261):
 * status 0 = found (binned by estimate), 1 = cold, 2 = estimate above
 * rd_cap (last bin), 3 = max_scan reached. hll_p <= 0 means 12; it is
 * clamped to [4, 14]. stats_host[4] = {found, cold, large, unresolved}.
 * est/status/pos (device, `samples` entries each) are optional outputs.
 * Synchronises `stream`. */
int mr_rd_hist_sampled(const int32_t* stream_dev, int32_t nnz, int32_t samples, int32_t sector_size,
                       int32_t rd_cap, int32_t hll_p, int32_t max_scan, uint32_t seed,
                       const int32_t* edges_host, int32_t nedges, int64_t* counts_host, int64_t* stats_host,
                       float* est_dev, int32_t* status_dev, int32_t* pos_dev, void* stream);

/* Sample seed of sampled_hll_rd_block_gpu (src/class.cu:1203). */
uint32_t mr_hll_seed(int32_t graph_id, int32_t stream_type);

/* ----------------------------------------------------------- predictor ---- */

typedef enum mr_model {
    MR_MODEL_MERBIT_SAMPLED = 0, /* include/model.cuh, ridge/out/merbit/sampled */
    MR_MODEL_MERBIT_EXACT = 1,   /* ridge/out/merbit/exact */
    MR_MODEL_CSR_SAMPLED = 2,    /* ridge/out/csr/sampled */
    MR_MODEL_CSR_EXACT = 3       /* ridge/out/csr/exact */
} mr_model;

/* exp(b + sum w_i r_i) over the 10 RD-bin probabilities. Replaces
 * rd_merbit_model::PredictSpeedup (include/model.cuh:91-94); returns
 * MR_ERR_PREDICT when the value is not finite or <= 0 (the reference throws,
 * src/class.cu:1317-1320). */
int mr_predict_speedup(int model, const double* features10, double* speedup);

/* Sampled RD (reference settings: sector 32, 30960 samples, p = 12,
 * max_scan 0, the 9 edges of src/class.cu:1267) + PredictSpeedup.
 * Replaces GRAPH::locality_predict (src/class.cu:1263-1326). features10 may
 * be NULL. */
int mr_locality_predict(const int32_t* stream_dev, int32_t nnz, int32_t ncols, int32_t graph_id,
                        double* features10, float* speedup, void* stream);

/* ------------------------------------------- predictor-gated reorder ---- */

typedef enum mr_gate {
    MR_GATE_SKIP = 0,      /* keep the current order */
    MR_GATE_RELABEL = 1,   /* reorder */
    MR_GATE_UNCERTAIN = 2  /* inside the band: the caller's policy decides */
} mr_gate;

/* Band gate of the ridge trainer (run_band_gate_scan, ridge/train.py:983-1026):
 * RELABEL when predicted >= tau_h, SKIP when predicted <= tau_l (SKIP wins
 * when both hold), UNCERTAIN otherwise. The trainer scans the pairs
 * (0.99, 1.01) ... (0.93, 1.07) (BAND_GATE_PAIRS, ridge/train.py:91-99). */
int mr_band_gate(double predicted_speedup, double tau_l, double tau_h, int32_t* decision);

/* Predicted reorder speedup of an x-access stream (colidx in CSR order) with
 * ridge model `model` (mr_model): the *_SAMPLED models take the sampled HLL
 * histogram of GRAPH::locality_predict (src/class.cu:1263-1311, seed from
 * graph_id), the *_EXACT models the exact histogram
 * (compute_sector_rd_histogram, src/class.cu:892-936); both with the
 * reference's 10 bins over 32-column sectors. features10 may be NULL.
 * Synchronises `stream`; MR_ERR_PREDICT as mr_predict_speedup. */
int mr_predict_reorder(const int32_t* stream_dev, int32_t nnz, int32_t ncols, int32_t graph_id, int32_t model,
                       double* features10, double* speedup, void* stream);

/* ------------------------------------------------------------- pGOrder ---- */

/* Partition size of gorder4: GRAPH::get_width (src/class.cu:733-750). */
int32_t mr_pgorder_width(int32_t n_rows, int64_t nnz);

/* pGOrder ordering on the host: perm_new2old[new] = old, bit-identical to
 * GRAPH::gorder4's order_on_cpu tasks (src/class.cu:2608-2690, :2220-2314,
 * include/integer_heap.cuh). A is a square host CSR with sorted columns.
 * vsize <= 0 uses mr_pgorder_width; threads <= 0 uses all cores. */
int mr_pgorder(int32_t n, const int32_t* rowptr_host, const int32_t* colidx_host, int32_t vsize,
               int32_t width, int32_t threads, uint32_t* perm_new2old_host);

/* ------------------------------------- other permutation producers ---- */

/* The reference's comparators for pGOrder, on the GPU; each writes
 * perm[old] = new (n = A->n_rows entries, device) for mr_permute_csr.
 * Degree of v = number of nonzeros in column v (the reference counts its
 * row_ind, which holds our column indices). Synchronise `stream`. */
/* Decreasing degree, ties by increasing id: GRAPH::relabel_degree
 * (src/class.cu:1493-1549). */
int mr_order_degree(const mr_csr_view* A, int32_t* perm_old2new_dev, void* stream);
/* Degree-based grouping: class ceilf(log2(degree + 1.0)) decreasing, ids
 * increasing within a class: GRAPH::dbg (src/class.cu:1660-1760). */
int mr_order_dbg(const mr_csr_view* A, int32_t* perm_old2new_dev, void* stream);
/* GRAPH::relabel_random (src/class.cu:1460-1491): the permutation the
 * reference's thrust::shuffle of the identity draws with
 * thrust::default_random_engine seeded with `seed` (the reference passes
 * graph_id), bit for bit. */
int mr_order_random(int32_t n, uint32_t seed, int32_t* perm_old2new_dev, void* stream);

/* pGOrder on the GPU: the same permutation as mr_pgorder (bit for bit), one
 * warp per block of vsize ids with its bucket queue in shared memory; A is a
 * square device CSR. vsize <= 0 uses mr_pgorder_width. Returns
 * MR_ERR_UNSUPPORTED (nothing written) when vsize > 32767, when
 * width * (sqrt(n)/4) exceeds the 16-bit key range, or when repeated
 * entries drive a key past it; use mr_pgorder then. Synchronises `stream`.
 * No reference counterpart (the reference orders on host threads,
 * GRAPH::gorder4, src/class.cu:2647-2683). */
int mr_pgorder_gpu(const mr_csr_view* A, int32_t vsize, int32_t width, uint32_t* perm_new2old_dev, void* stream);

/* ------------------------------------------ GRAPH-style host object ---- */

/* A square matrix resident on the device with its current permutation
 * (perm[old] = new), mirroring GRAPH<float> (include/class.cuh:58-97). */
typedef struct mr_graph mr_graph;

int mr_graph_create(int32_t n, int64_t nnz, const int32_t* rowptr_host, const int32_t* colidx_host,
                    const void* vals_host, int32_t dtype, int32_t graph_id, mr_graph** g);
int mr_graph_destroy(mr_graph* g);
/* GRAPH::gorder4(env, vsize, width) (src/class.cu:2608-2722): host pGOrder,
 * then the device relabel; ms_order/ms_relabel may be NULL. */
int mr_graph_gorder4(mr_graph* g, int32_t vsize, int32_t width, double* ms_order, double* ms_relabel);
/* GRAPH::locality_predict (src/class.cu:1263-1326) on the current order. */
int mr_graph_locality_predict(mr_graph* g, double* features10, float* speedup);
/* GRAPH::spmv(env, method) (src/class.cu:1331-1454): method "csr" or
 * "merbit"; runs `iters` SpMVs with x = x_host (original numbering, NULL =
 * all ones as the reference) and returns y in the original numbering.
 * ms_plan/ms_spmv may be NULL (ms_spmv is per SpMV). */
int mr_graph_spmv(mr_graph* g, const char* method, int32_t iters, const float* x_host, float* y_host,
                  double* ms_plan, double* ms_spmv);
/* Predictor-gated reorder (the pipeline sampled RD -> PredictSpeedup -> band
 * gate -> reorder-or-skip): mr_predict_reorder on the current order with
 * `model`, mr_band_gate(tau_l, tau_h), then mr_graph_gorder4(vsize, width)
 * when the gate says RELABEL, or UNCERTAIN and relabel_uncertain != 0.
 * decision (mr_gate) and predicted may be NULL. */
int mr_graph_gated_reorder(mr_graph* g, int32_t model, double tau_l, double tau_h, int32_t relabel_uncertain,
                           int32_t vsize, int32_t width, int32_t* decision, double* predicted);
/* Current permutation perm[old] = new, and the current device CSR view. */
int mr_graph_get_perm(const mr_graph* g, int32_t* perm_host);
int mr_graph_view(const mr_graph* g, mr_csr_view* view);

#ifdef __cplusplus
}
#endif
#endif /* MR_H */
