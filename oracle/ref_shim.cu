/*
 * C-ABI shim around the reference's own code (Zhangq388/MATRIX-REORDER).
 *
 * TEST INFRASTRUCTURE ONLY. oracle/build_ref.sh compiles this file together
 * with the reference's src/class.cu, pulled in by path from the reference
 * checkout (REF_CLASS_CU), into oracle/_ref/libmr_ref.so. Nothing of the
 * reference is copied here: the shim only calls the reference's functions
 * and kernels so that tests can compare the product against them.
 *
 * Host-only entry points (run in any container): ref_get_width,
 * ref_rd_hist_exact, ref_pgorder_host, ref_predict, ref_shuffle_host.
 * Device entry points (need a GPU): ref_tile_build, ref_merbit_spmv,
 * ref_hll_sampled, ref_relabel_sort, ref_gorder4_full, ref_relabel_order, ref_cusparse_spmv.
 *
 * Index convention: the reference's `col_ind` is our row and its `row_ind`
 * is our column (src/class.cu:445-454, :1342, :1372).
 */
#include REF_CLASS_CU

std::fstream FSTR;

extern "C" {

int ref_get_width(int nrow, int nnz)
{
    GRAPH<float> g;
    g.nrow = nrow;
    g.nnz = nnz;
    return g.get_width(); /* src/class.cu:733-750 */
}

/* compute_sector_rd_histogram (src/class.cu:892-936) over the access stream,
 * i.e. our colidx in CSR order. probs has nedges+1 entries. */
void ref_rd_hist_exact(const int* stream, int nrow, int nnz, int sector_size,
                       const int* edges, int nedges, double* probs)
{
    std::vector<int> e(edges, edges + nedges);
    std::vector<double> out;
    compute_sector_rd_histogram(stream, nrow, nnz, sector_size, e, out);
    for (int i = 0; i <= nedges; ++i) probs[i] = out[i];
}

/* The host part of GRAPH::gorder4 (src/class.cu:2647-2683): one order_on_cpu
 * task per vsize block on a ThreadPool(128). off1/ind1 = the reference's
 * sort(true) CSR (our columns), off2/ind2 = sort(false) CSR (our rows). */
void ref_pgorder_host(int nrow, const int* off1, const int* ind1, const int* off2,
                      const int* ind2, int vsize, int width, unsigned int* h_perm)
{
    std::iota(h_perm, h_perm + nrow, 0);
    std::vector<std::unique_ptr<Node>> NODE(nrow);
    for (int i = 0; i < nrow; ++i) NODE[i] = std::make_unique<Node>(i);
    int maxiter = (nrow + vsize - 1) / vsize;
    ThreadPool pool(128);
    std::vector<std::future<void>> futures;
    int L = std::sqrt(nrow) / 4;
    for (int b = 0; b < maxiter; ++b) {
        int start = b * vsize;
        int len = (start + vsize < nrow) ? vsize : nrow - start;
        futures.emplace_back(pool.enqueue([&NODE, off1, ind1, off2, ind2, h_perm, start, b, len, width, L]() {
            order_on_cpu(&NODE, off1, ind1, off2, ind2, &h_perm[start], b, len, width, L);
        }));
    }
    for (auto& f : futures) f.get();
}

/* local_swap (src/class.cu:236-301) on an identity-initialised permutation. */
void ref_local_swap(int nrow, float rho, int near_, int window, unsigned long long seed, int* permutation)
{
    local_swap(nrow, rho, near_, window, seed, permutation);
}

double ref_predict(const double* r10)
{
    std::array<double, rd_merbit_model::kFeatureCount> a{};
    for (int i = 0; i < 10; ++i) a[i] = r10[i];
    return rd_merbit_model::PredictSpeedup(a); /* include/model.cuh:91-94 */
}

/* ------------------------------------------------------------- device -- */

/* Tile_Kernel<256,14> (include/merbit.cuh:55-155) into caller buffers:
 * tile_x/tile_y[tile_num+1], desc[lane_num] (32-bit words). */
int ref_tile_build(const int* d_rowptr, int nrow, int nnz, unsigned int* tile_x,
                   unsigned int* tile_y, unsigned int* desc)
{
    const int lane_num = (nrow + nnz + 14 - 1) / 14;
    const int tile_num = (lane_num + 31) / 32;
    cudaMemset(tile_x, 0, sizeof(unsigned int) * (tile_num + 1));
    cudaMemset(tile_y, 0, sizeof(unsigned int) * (tile_num + 1));
    cudaMemset(desc, 0, sizeof(unsigned int) * lane_num);
    const int grid = (lane_num + 256) / 256;
    Tile_Kernel<256, 14><<<grid, 256>>>(d_rowptr, nrow, nnz, tile_num, lane_num, tile_x, tile_y, desc);
    return (int)cudaDeviceSynchronize();
}

/* `iters` launches of merbit_kernel<float,256,14> exactly as GRAPH::spmv
 * drives it (src/class.cu:1419-1427), y/z ping-pong included. The final
 * result is left in y. Returns the CUDA status; *ms gets the mean time per
 * launch from CUDA events. */
int ref_merbit_spmv(const int* d_rowptr, const int* d_colidx, const float* d_vals, int nrow, int nnz,
                    const unsigned int* tile_x, const unsigned int* tile_y, const unsigned int* desc,
                    const float* d_x, float* d_y, float* d_z, int iters, float* ms)
{
    const int lane_num = (nrow + nnz + 14 - 1) / 14;
    const int tile_num = (lane_num + 31) / 32;
    const int grid = (lane_num + 256 - 1) / 256;
    cudaMemset(d_y, 0, sizeof(float) * nrow);
    cudaMemset(d_z, 0, sizeof(float) * nrow);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float* y = d_y;
    float* z = d_z;
    cudaEventRecord(a);
    for (int r = 0; r < iters; ++r) {
        merbit_kernel<float, 256, 14><<<grid, 256>>>(d_rowptr, d_colidx, d_vals, nrow, nnz, tile_x, tile_y,
                                                     desc, tile_num, lane_num, d_x, y, z);
        std::swap(y, z);
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    if (ms) *ms = t / (iters > 0 ? iters : 1);
    if (z != d_y) cudaMemcpy(d_y, z, sizeof(float) * nrow, cudaMemcpyDeviceToDevice);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return (int)cudaDeviceSynchronize();
}

/* sampled_hll_rd_block_kernel (src/class.cu:1014-1131) launched as
 * sampled_hll_rd_block_gpu does (:1186-1206). */
int ref_hll_sampled(const int* d_stream, int nnz, int samples, int sector_size, unsigned int seed,
                    int rd_cap, int max_scan, int hll_p, float* d_est, int* d_status, int* d_pos)
{
    const int hll_m = 1 << hll_p;
    const size_t smem = sizeof(int) * (size_t)hll_m;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(sampled_hll_rd_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    sampled_hll_rd_block_kernel<<<samples, 256, smem>>>(d_stream, nnz, samples, sector_size, seed, rd_cap,
                                                        max_scan, hll_p, hll_m, d_est, d_status, d_pos);
    return (int)cudaDeviceSynchronize();
}

/* The reference relabel: gather both index arrays through perm, then
 * GRAPH::sort(false) (src/class.cu:2699-2705, :423-457). d_row_ind holds our
 * columns and d_col_ind our rows, as the reference stores them. */
int ref_relabel_sort(int nrow, int nnz, int* d_row_ind, int* d_col_ind, float* d_vals, const int* d_perm)
{
    thrust::device_ptr<int> r(d_row_ind), c(d_col_ind);
    thrust::device_ptr<const int> p(d_perm);
    thrust::gather(r, r + nnz, p, r);
    thrust::gather(c, c + nnz, p, c);
    GRAPH<float> g;
    g.nrow = nrow;
    g.nnz = nnz;
    g.row_ind = d_row_ind;
    g.col_ind = d_col_ind;
    g.values = d_vals;
    g.sort(false);
    g.row_ind = nullptr;
    g.col_ind = nullptr;
    g.values = nullptr;
    return (int)cudaDeviceSynchronize();
}

/* The whole GRAPH::gorder4 (src/class.cu:2608-2722) on device COO arrays:
 * builds both CSRs with cuSPARSE, orders on the host, relabels and sorts.
 * perm_out[old] = new afterwards. */
int ref_gorder4_full(int nrow, int nnz, int* d_row_ind, int* d_col_ind, float* d_vals, int vsize, int width,
                     int* h_perm_out)
{
    ENV env(0, "", "");
    // ENV always selects device 1 (include/class.cuh:23); on a one-GPU box
    // that fails and leaves an error that Thrust would report later
    cudaSetDevice(0);
    cudaGetLastError();
    GRAPH<float> g;
    g.nrow = nrow;
    g.nnz = nnz;
    g.row_ind = d_row_ind;
    g.col_ind = d_col_ind;
    g.values = d_vals;
    cudaMalloc((void**)&g.perm, sizeof(int) * nrow);
    g.gorder4(env, vsize, width);
    cudaMemcpy(h_perm_out, g.perm, sizeof(int) * nrow, cudaMemcpyDeviceToHost);
    cudaFree(g.perm);
    g.perm = nullptr;
    g.row_ind = nullptr;
    g.col_ind = nullptr;
    g.values = nullptr;
    return (int)cudaDeviceSynchronize();
}

/* GRAPH::relabel_degree (kind 0, src/class.cu:1493-1549), GRAPH::dbg (kind 1,
 * :1660-1760) or GRAPH::relabel_random (kind 2, :1460-1491) on COO arrays
 * (row_ind = our column indices, col_ind = our row indices); perm starts as
 * the identity, as GRAPH's constructors leave it. The COO arrays are
 * relabelled in place by the reference. h_perm_out[old] = new. */
int ref_relabel_order(int kind, int nrow, int nnz, int* d_row_ind, int* d_col_ind, float* d_vals, int graph_id,
                      int* h_perm_out)
{
    ENV env(0, "", "");
    cudaSetDevice(0);  // see ref_gorder4_full
    cudaGetLastError();
    GRAPH<float> g;
    g.nrow = nrow;
    g.nnz = nnz;
    g.graph_id = graph_id;
    g.row_ind = d_row_ind;
    g.col_ind = d_col_ind;
    g.values = d_vals;
    cudaMalloc((void**)&g.perm, sizeof(int) * nrow);
    thrust::sequence(thrust::device_ptr<int>(g.perm), thrust::device_ptr<int>(g.perm) + nrow);
    if (kind == 0)
        g.relabel_degree();
    else if (kind == 1)
        g.dbg(env);
    else
        g.relabel_random();
    cudaMemcpy(h_perm_out, g.perm, sizeof(int) * nrow, cudaMemcpyDeviceToHost);
    cudaFree(g.perm);
    g.perm = nullptr;
    g.row_ind = nullptr;
    g.col_ind = nullptr;
    g.values = nullptr;
    return (int)cudaDeviceSynchronize();
}

/* cuSPARSE CSR_ALG1 SpMV, the reference's plain-CSR path (src/class.cu:1359-1397),
 * timed over `iters` launches with CUDA events. */
int ref_cusparse_spmv(const int* d_rowptr, const int* d_colidx, const float* d_vals, int nrow, int nnz,
                      const float* d_x, float* d_y, int iters, float* ms)
{
    cusparseHandle_t h;
    cusparseCreate(&h);
    cusparseSpMatDescr_t A;
    cusparseDnVecDescr_t X, Y;
    cusparseCreateCsr(&A, nrow, nrow, nnz, (void*)d_rowptr, (void*)d_colidx, (void*)d_vals, CUSPARSE_INDEX_32I,
                      CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F);
    cusparseCreateDnVec(&X, nrow, (void*)d_x, CUDA_R_32F);
    cusparseCreateDnVec(&Y, nrow, (void*)d_y, CUDA_R_32F);
    float alpha = 1.f, beta = 0.f;
    size_t bs = 0;
    void* buf = nullptr;
    cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, X, &beta, Y, CUDA_R_32F,
                            CUSPARSE_SPMV_CSR_ALG1, &bs);
    cudaMalloc(&buf, bs > 0 ? bs : 16);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, X, &beta, Y, CUDA_R_32F, CUSPARSE_SPMV_CSR_ALG1, buf);
    cudaEventRecord(a);
    for (int r = 0; r < iters; ++r)
        cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, X, &beta, Y, CUDA_R_32F,
                     CUSPARSE_SPMV_CSR_ALG1, buf);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    if (ms) *ms = t / (iters > 0 ? iters : 1);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    cusparseDestroySpMat(A);
    cusparseDestroyDnVec(X);
    cusparseDestroyDnVec(Y);
    cusparseDestroy(h);
    return (int)cudaDeviceSynchronize();
}

/* The permutation GRAPH::relabel_random draws (src/class.cu:1467-1473):
 * thrust::shuffle of the identity with thrust::default_random_engine seeded
 * with graph_id, here run by Thrust's host backend (the same generic
 * algorithm as the device call) so that fixtures can be made without a GPU.
 * out[old] = new. */
int ref_shuffle_host(int n, unsigned int seed, int* out)
{
    thrust::host_vector<int> v(n);
    thrust::sequence(thrust::host, v.begin(), v.end());
    thrust::default_random_engine rng;
    rng.seed(seed);
    thrust::shuffle(thrust::host, v.begin(), v.end(), rng);
    for (int i = 0; i < n; ++i) out[i] = v[i];
    return 0;
}

} /* extern "C" */
