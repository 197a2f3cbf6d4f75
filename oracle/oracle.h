/*
 * CPU oracle for the reordered-SpMV path of Zhangq388/MATRIX-REORDER.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, in plain C, the reference's
 * algorithms for the hot path so that tests (and bench.py's CPU-baseline leg)
 * can check the CUDA product against it. The product library never links,
 * loads or calls anything here.
 *
 * Convention: matrices are textbook CSR (rowptr[n+1], colidx[nnz], vals[nnz]).
 * The reference stores the same matrix transposed (its `col_ind` is our row and
 * its `row_ind` is our column, src/class.cu:445-454, :1342, :1372).
 *
 * Parity pin: every function here is checked against the reference's own code
 * compiled from its sources (oracle/build_ref.sh -> oracle/_ref/) and against
 * fixtures in tests/golden/ produced from that build.
 */
#ifndef MR_ORACLE_H
#define MR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = A x accumulated in FP64 (the numerical oracle for every SpMV test). */
void orc_spmv_csr_f64(int n, const int32_t* rowptr, const int32_t* colidx,
                      const float* vals, const float* x, double* y);

/* y = A x in FP32 with OpenMP over rows: the timed CPU baseline. The reference
 * has no CPU SpMV; this is the plain restatement of CSR SpMV. Returns the
 * number of threads used. */
int orc_spmv_csr_f32_omp(int n, const int32_t* rowptr, const int32_t* colidx,
                         const float* vals, const float* x, float* y, int threads);

/* MERBIT plan (include/merbit.cuh:24-155). Writes tile_x/tile_y[tile_num+1]
 * and lane_desc[lane_num] (64-bit container; the reference stores 32-bit words
 * when sigma < 15). Returns 0, or -1 on bad arguments. */
int orc_merbit_plan(const int32_t* rowptr, int nrow, int nnz, int sigma,
                    uint32_t* tile_x, uint32_t* tile_y, uint64_t* lane_desc);
void orc_merbit_sizes(int nrow, int nnz, int sigma, int* lane_num, int* tile_num);

/* Symmetric permutation B = P A P^T with B[perm[r], perm[c]] = A[r, c],
 * columns sorted within each row, ties kept in source order
 * (src/class.cu:2688-2705 with GRAPH::sort(false), src/class.cu:423-457). */
void orc_permute_csr(int n, const int32_t* rowptr, const int32_t* colidx,
                     const float* vals, const int32_t* perm_old2new,
                     int32_t* out_rowptr, int32_t* out_colidx, float* out_vals);

/* Exact sector reuse-distance histogram (src/class.cu:864-936).
 * counts[nedges+1] and *valid receive integer counts. */
void orc_rd_hist_exact(const int32_t* stream, int64_t nnz, int ncols, int sector_size,
                       const int32_t* edges, int nedges, int64_t* counts, int64_t* valid);

/* Sampled HyperLogLog reuse distance (src/class.cu:954-1131), simulated
 * sequentially. Per sample: est, status, pos as the reference kernel writes. */
void orc_hll_sampled(const int32_t* stream, int nnz, int samples, int sector_size,
                     uint32_t seed, int rd_cap, int max_scan, int hll_p,
                     float* est, int32_t* status, int32_t* pos);
/* Host binning of the per-sample results (src/class.cu:1213-1256). */
void orc_hll_bin(int samples, const float* est, const int32_t* status,
                 const int32_t* edges, int nedges, int64_t* counts,
                 int64_t* found, int64_t* cold, int64_t* large, int64_t* unresolved);

/* pGOrder (gorder4): src/class.cu:2608-2722 with order_on_cpu :2220-2314 and
 * Integer_Heap include/integer_heap.cuh. perm_new2old[new] = old. */
void orc_pgorder(int n, const int32_t* rowptr, const int32_t* colidx,
                 int vsize, int width, uint32_t* perm_new2old);
int orc_get_width(int nrow, int nnz);

/* exp(intercept + sum coef_i * r_i) (include/model.cuh:84-95). */
double orc_predict(const double* coef10, double intercept, const double* r10);

/* GRAPH::relabel_random (src/class.cu:1460-1491): perm_old2new = the
 * identity shuffled by thrust::shuffle with thrust::default_random_engine
 * seeded with graph_id. The algorithm is Thrust's (CCCL bundled with CUDA
 * 12.9, thrust/system/detail/generic/shuffle.inl): a 24-round Feistel
 * bijection over the next power of two >= n, compacted to [0, n) in index
 * order. */
void orc_order_random(int n, uint32_t seed, int32_t* perm_old2new);

#ifdef __cplusplus
}
#endif
#endif
