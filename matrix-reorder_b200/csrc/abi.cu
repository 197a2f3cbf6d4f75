// extern "C" entry points of libmr: argument checks, plan ownership and
// dispatch to the kernels. Declared in include/mr.h.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace mr {

static thread_local std::string g_last_error;

void note_cuda_error(cudaError_t e, const char* what, const char* file, int line)
{
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
    g_last_error = buf;
}

void note_error(const char* msg) { g_last_error = msg ? msg : ""; }

cudaMemPool_t scratch_pool()
{
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= dev) pools.resize((size_t)dev + 1, nullptr);
    if (!pools[(size_t)dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;  // callers fall back to the default pool
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[(size_t)dev] = p;
    }
    return pools[(size_t)dev];
}

static int check_view(const mr_csr_view* A, bool need_square)
{
    if (!A) return MR_ERR_INVALID_ARG;
    if (A->n_rows < 0 || A->n_cols < 0 || A->nnz < 0 || A->nnz > INT32_MAX) return MR_ERR_INVALID_ARG;
    if (A->dtype != MR_F32 && A->dtype != MR_F16 && A->dtype != MR_BF16) return MR_ERR_UNSUPPORTED;
    if (!A->rowptr) return MR_ERR_INVALID_ARG;
    if (A->nnz > 0 && (!A->colidx || !A->vals)) return MR_ERR_INVALID_ARG;
    if (need_square && A->n_rows != A->n_cols) return MR_ERR_INVALID_ARG;
    return MR_OK;
}

}  // namespace mr

using namespace mr;


extern "C" {

const char* mr_status_string(int s)
{
    switch (s) {
    case MR_OK: return "ok";
    case MR_ERR_INVALID_ARG: return "invalid argument";
    case MR_ERR_CUDA: return "CUDA error";
    case MR_ERR_NOMEM: return "out of memory";
    case MR_ERR_INVALID_PERM: return "permutation is not a bijection";
    case MR_ERR_UNSUPPORTED: return "unsupported dtype or option";
    case MR_ERR_TIMEOUT: return "bounded wait expired";
    case MR_ERR_BUSY: return "admission refused";
    case MR_ERR_NOT_FOUND: return "unknown id";
    case MR_ERR_INTERNAL: return "internal consistency check failed";
    case MR_ERR_PREDICT: return "predictor returned an invalid speedup";
    default: return "unknown status";
    }
}

int mr_version(void) { return 10000; }

int mr_release_scratch(void)
{
    cudaMemPool_t p = scratch_pool();
    if (!p) return MR_ERR_CUDA;
    MR_CUDA_TRY(cudaDeviceSynchronize());
    MR_CUDA_TRY(cudaMemPoolTrimTo(p, 0));
    return MR_OK;
}

const char* mr_last_error(void) { return g_last_error.c_str(); }

int mr_spmv_csr(const mr_csr_view* A, const float* x, float* y, void* stream)
{
    MR_TRY(check_view(A, false));
    if (A->n_rows > 0 && (!y || (A->nnz > 0 && !x))) return MR_ERR_INVALID_ARG;
    return launch_csr_spmv(A->n_rows, A->nnz, A->rowptr, A->colidx, A->vals, A->dtype, x, y, as_stream(stream));
}

int mr_merbit_plan_create(const mr_csr_view* A, int sigma, int block, void* stream, mr_merbit_plan** out)
{
    return mr_merbit_plan_create_ex(A, sigma, block, 0, stream, out);
}

int mr_merbit_plan_create_ex(const mr_csr_view* A, int sigma, int block, int flags, void* stream,
                             mr_merbit_plan** out)
{
    if (!out) return MR_ERR_INVALID_ARG;
    *out = nullptr;
    MR_TRY(check_view(A, false));
    if (sigma == 0) sigma = 14;
    if (block == 0) block = 1024;
    if (sigma < 1 || sigma > 42) return MR_ERR_INVALID_ARG;
    if (block != 128 && block != 256 && block != 512 && block != 1024) return MR_ERR_UNSUPPORTED;
    const int64_t items = (int64_t)A->n_rows + A->nnz;
    if (items + 32ll * sigma * 257 > (int64_t)INT32_MAX) return MR_ERR_INVALID_ARG;
    {
        int ok = 0;
        MR_TRY(validate_csr(*A, &ok, as_stream(stream)));
        if (!ok) return MR_ERR_INVALID_ARG;
    }
    auto* h = new (std::nothrow) mr_merbit_plan;
    if (!h) return MR_ERR_NOMEM;
    MerbitPlan& p = h->p;
    p.sigma = sigma;
    p.block = block;
    p.n_rows = A->n_rows;
    p.nnz = A->nnz;
    p.lane_num = (int)((items + sigma - 1) / sigma);
    p.tile_num = (p.lane_num + 31) / 32;
    cudaGetDevice(&p.device);
    const size_t desc_bytes = sigma < 15 ? 4 : 8;
    cudaStream_t st = as_stream(stream);
    auto fail = [&](int code) {
        free_plan_buffers(p);
        delete h;
        return code;
    };
    if (cudaMalloc(&p.tile_x, sizeof(uint32_t) * ((size_t)p.tile_num + 1)) != cudaSuccess ||
        cudaMalloc(&p.tile_y, sizeof(uint32_t) * ((size_t)p.tile_num + 1)) != cudaSuccess ||
        cudaMalloc(&p.lane_desc, desc_bytes * (size_t)std::max(p.lane_num, 1)) != cudaSuccess ||
        cudaMalloc(&p.carry, sizeof(float) * (size_t)std::max(p.tile_num, 1)) != cudaSuccess ||
        cudaMalloc(&p.ticket, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return fail(MR_ERR_NOMEM);
    }
    if (cudaMemsetAsync(p.ticket, 0, sizeof(int), st) != cudaSuccess) return fail(MR_ERR_CUDA);
    int s = launch_merbit_plan(A->rowptr, A->n_rows, (int)A->nnz, sigma, p.lane_num, p.tile_num, p.tile_x, p.tile_y,
                               p.lane_desc, st);
    if (s != MR_OK) return fail(s);
    p.gather_mode = (flags & MR_PLAN_GATHER_NO_L1) ? 1 : (flags & MR_PLAN_GATHER_L2_ONLY) ? 2 : 0;
    if (flags & MR_PLAN_SMALL_HUB_CACHE) p.hub_limit = 8192;
    if ((flags >> 8) & 0xffff) p.hub_limit = 1024 * ((flags >> 8) & 0xffff);
    if (block == 1024 && !(flags & MR_PLAN_NO_HUB_CACHE)) {
        s = build_hub_cache(p, *A, st);
        if (s != MR_OK) return fail(s);
    }
    if (block == 1024) {
        s = build_chunk_bounds(p, A->colidx, st);
        if (s != MR_OK) return fail(s);
    }
    *out = h;
    return MR_OK;
}

int mr_merbit_plan_destroy(mr_merbit_plan* h)
{
    if (!h) return MR_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != h->p.device) cudaSetDevice(h->p.device);
    cudaDeviceSynchronize();
    free_plan_buffers(h->p);
    if (dev != h->p.device) cudaSetDevice(dev);
    delete h;
    return MR_OK;
}

int mr_merbit_plan_get_info(const mr_merbit_plan* h, mr_merbit_plan_info* info)
{
    if (!h || !info) return MR_ERR_INVALID_ARG;
    const MerbitPlan& p = h->p;
    info->sigma = p.sigma;
    info->block = p.block;
    info->n_rows = p.n_rows;
    info->nnz = p.nnz;
    info->lane_num = p.lane_num;
    info->tile_num = p.tile_num;
    info->desc_bytes = p.sigma < 15 ? 4 : 8;
    info->tile_x_dev = p.tile_x;
    info->tile_y_dev = p.tile_y;
    info->lane_desc_dev = p.lane_desc;
    info->hub_columns = p.hub_k;
    info->hub_coverage = p.hub_coverage;
    return MR_OK;
}

int mr_spmv_merbit(const mr_merbit_plan* h, const mr_csr_view* A, const float* x, float* y, void* stream)
{
    if (!h) return MR_ERR_INVALID_ARG;
    MR_TRY(check_view(A, false));
    const MerbitPlan& p = h->p;
    if (A->n_rows != p.n_rows || A->nnz != p.nnz) return MR_ERR_INVALID_ARG;
    if (!merbit_sigma_supported(p.sigma)) return MR_ERR_UNSUPPORTED;
    if (p.n_rows > 0 && (!y || (p.nnz > 0 && !x))) return MR_ERR_INVALID_ARG;
    return launch_merbit_spmv(p, A->colidx, A->vals, A->dtype, x, y, p.carry, as_stream(stream));
}

int mr_permute_csr(const mr_csr_view* A, const int32_t* perm, int32_t* out_rowptr, int32_t* out_colidx,
                   void* out_vals, void* stream)
{
    MR_TRY(check_view(A, true));
    if (!perm && A->n_rows > 0) return MR_ERR_INVALID_ARG;
    if (!out_rowptr || (A->nnz > 0 && (!out_colidx || !out_vals))) return MR_ERR_INVALID_ARG;
    return permute_csr(*A, perm, out_rowptr, out_colidx, out_vals, as_stream(stream));
}

int mr_permute_vector(int32_t n, const int32_t* perm, const float* in, float* out, int inverse, void* stream)
{
    if (n < 0 || (n > 0 && (!perm || !in || !out))) return MR_ERR_INVALID_ARG;
    return launch_permute_vector(n, perm, in, out, inverse, as_stream(stream));
}

int mr_perm_invert(int32_t n, const int32_t* perm, int32_t* inv, void* stream)
{
    if (n < 0 || (n > 0 && (!perm || !inv))) return MR_ERR_INVALID_ARG;
    if (n == 0) return MR_OK;
    cudaStream_t st = as_stream(stream);
    DevBuf flag;
    MR_TRY(flag.alloc(sizeof(int), st));
    MR_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    MR_TRY(launch_perm_invert(n, perm, inv, flag.as<int>(), st));
    int h = 0;
    MR_CUDA_TRY(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    return h ? MR_ERR_INVALID_PERM : MR_OK;
}

int mr_csr_validate(const mr_csr_view* A, int* valid, void* stream)
{
    if (!valid) return MR_ERR_INVALID_ARG;
    MR_TRY(check_view(A, false));
    return validate_csr(*A, valid, as_stream(stream));
}

int mr_check_perm(const int32_t* perm, int32_t n, int* valid, void* stream)
{
    if (!valid || n < 0 || (n > 0 && !perm)) return MR_ERR_INVALID_ARG;
    return check_perm(perm, n, valid, as_stream(stream));
}

static int check_edges(const int32_t* edges, int32_t nedges)
{
    if (!edges || nedges < 1 || nedges > 63) return MR_ERR_INVALID_ARG;
    for (int i = 1; i < nedges; ++i)
        if (edges[i] < edges[i - 1]) return MR_ERR_INVALID_ARG;
    return MR_OK;
}

int mr_rd_hist_exact(const int32_t* s, int64_t nnz, int32_t ncols, int32_t sector, const int32_t* edges,
                     int32_t nedges, int64_t* counts, int64_t* valid, void* stream)
{
    if (nnz < 0 || nnz > INT32_MAX || ncols < 0 || sector <= 0 || !counts || !valid || (nnz > 0 && !s))
        return MR_ERR_INVALID_ARG;
    MR_TRY(check_edges(edges, nedges));
    return rd_hist_exact(s, nnz, ncols, sector, edges, nedges, counts, valid, as_stream(stream));
}

int mr_rd_hist_sampled(const int32_t* s, int32_t nnz, int32_t samples, int32_t sector, int32_t rd_cap, int32_t hll_p,
                       int32_t max_scan, uint32_t seed, const int32_t* edges, int32_t nedges, int64_t* counts,
                       int64_t* stats, float* est, int32_t* status, int32_t* pos, void* stream)
{
    // argument rules of sampled_hll_rd_block_gpu (src/class.cu:1149-1167)
    if (!counts || !stats || nnz < 0 || (nnz > 1 && !s)) return MR_ERR_INVALID_ARG;
    if (sector <= 0) return MR_ERR_INVALID_ARG;
    MR_TRY(check_edges(edges, nedges));
    if (rd_cap > 0 && rd_cap < edges[nedges - 1]) return MR_ERR_INVALID_ARG;
    return rd_hist_sampled(s, nnz, samples, sector, rd_cap, hll_p, max_scan, seed, edges, nedges, counts, stats, est,
                           status, pos, as_stream(stream));
}

int mr_pgorder_gpu(const mr_csr_view* A, int32_t vsize, int32_t width, uint32_t* perm, void* stream)
{
    MR_TRY(check_view(A, true));
    if (!perm && A->n_rows > 0) return MR_ERR_INVALID_ARG;
    if (width < 1) return MR_ERR_INVALID_ARG;
    return pgorder_gpu(A->n_rows, A->rowptr, A->colidx, (int32_t)A->nnz, vsize, width, perm, as_stream(stream));
}

int mr_band_gate(double predicted, double tau_l, double tau_h, int32_t* decision)
{
    if (!decision || !(tau_l == tau_l) || !(tau_h == tau_h)) return MR_ERR_INVALID_ARG;
    // run_band_gate_scan (ridge/train.py:993-995): "relabel" is set first,
    // "skip" second, so skip wins when both thresholds hold
    int32_t d = MR_GATE_UNCERTAIN;
    if (predicted >= tau_h) d = MR_GATE_RELABEL;
    if (predicted <= tau_l) d = MR_GATE_SKIP;
    *decision = d;
    return MR_OK;
}

int mr_predict_reorder(const int32_t* s, int32_t nnz, int32_t ncols, int32_t graph_id, int32_t model,
                       double* features10, double* speedup, void* stream)
{
    static const int32_t kEdges[9] = {1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824};
    if (!speedup || ncols < 0 || nnz < 0) return MR_ERR_INVALID_ARG;
    if (model != MR_MODEL_MERBIT_SAMPLED && model != MR_MODEL_MERBIT_EXACT && model != MR_MODEL_CSR_SAMPLED &&
        model != MR_MODEL_CSR_EXACT)
        return MR_ERR_INVALID_ARG;
    double f[10];
    int64_t counts[10];
    if (model == MR_MODEL_MERBIT_SAMPLED || model == MR_MODEL_CSR_SAMPLED) {
        // settings of GRAPH::locality_predict (src/class.cu:1265-1277)
        int64_t stats[4];
        MR_TRY(mr_rd_hist_sampled(s, nnz, 30960, 32, kEdges[8], 12, 0, mr_hll_seed(graph_id, 0), kEdges, 9, counts,
                                  stats, nullptr, nullptr, nullptr, stream));
        const int64_t valid = stats[0] + stats[2];  // found + large
        for (int i = 0; i < 10; ++i) f[i] = valid > 0 ? (double)counts[i] / (double)valid : 0.0;
    } else {
        // the exact branch of locality_predict (src/class.cu:1284-1298)
        int64_t valid = 0;
        MR_TRY(mr_rd_hist_exact(s, nnz, ncols, 32, kEdges, 9, counts, &valid, stream));
        for (int i = 0; i < 10; ++i) f[i] = valid > 0 ? (double)counts[i] / (double)valid : 0.0;
    }
    if (features10)
        for (int i = 0; i < 10; ++i) features10[i] = f[i];
    return mr_predict_speedup(model, f, speedup);
}

int mr_locality_predict(const int32_t* s, int32_t nnz, int32_t ncols, int32_t graph_id, double* features10,
                        float* speedup, void* stream)
{
    // settings of GRAPH::locality_predict (src/class.cu:1265-1277)
    static const int32_t kEdges[9] = {1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824};
    if (!speedup || ncols < 0) return MR_ERR_INVALID_ARG;
    int64_t counts[10], stats[4];
    MR_TRY(mr_rd_hist_sampled(s, nnz, 30960, 32, kEdges[8], 12, 0, mr_hll_seed(graph_id, 0), kEdges, 9, counts, stats,
                              nullptr, nullptr, nullptr, stream));
    double f[10];
    const int64_t valid = stats[0] + stats[2];  // found + large
    for (int i = 0; i < 10; ++i) f[i] = valid > 0 ? (double)counts[i] / (double)valid : 0.0;
    if (features10)
        for (int i = 0; i < 10; ++i) features10[i] = f[i];
    double sp = 0.0;
    const int rc = mr_predict_speedup(MR_MODEL_MERBIT_SAMPLED, f, &sp);
    *speedup = (float)sp;
    return rc;
}

}  // extern "C"
