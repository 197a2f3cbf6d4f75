// mr_graph: host object mirroring the reference's GRAPH<float> operator API
// (include/class.cuh:58-97) on top of the libmr entry points.
//
// It keeps a square matrix resident on the device in its current order plus
// the composed permutation perm[original] = current, and offers the
// reference's three hot-path operations:
//   gorder4          (src/class.cu:2608-2722): pGOrder (on the GPU when its
//                    queue fits, else on host threads; the same permutation)
//                    + device relabel
//   locality_predict (src/class.cu:1263-1326): sampled RD + ridge predictor
//   spmv(method)     (src/class.cu:1331-1454): "csr" or "merbit" SpMV,
//                    returning y in the original numbering as the
//                    reference's check does (src/class.cu:1435-1445),
// plus the predictor-gated reorder (RD features -> ridge model -> band gate
// of ridge/train.py:983-1026 -> gorder4 or keep the order).
#include <chrono>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace mr;

struct mr_graph {
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t dtype = MR_F32;
    int32_t graph_id = 0;
    int32_t* rowptr = nullptr;
    int32_t* colidx = nullptr;
    void* vals = nullptr;
    int32_t* perm = nullptr;  // perm[original] = current
    cudaStream_t st = nullptr;

    mr_csr_view view() const { return {n, n, nnz, rowptr, colidx, vals, dtype}; }
};

namespace {

__global__ void iota_kernel(int32_t* p, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

// composed[i] = step[prev[i]]
__global__ void compose_kernel(const int32_t* __restrict__ step, int32_t* __restrict__ perm, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) perm[i] = step[perm[i]];
}

__global__ void fill_kernel(float* x, int n, float v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8)); }

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void free_graph(mr_graph* g)
{
    cudaFree(g->rowptr);
    cudaFree(g->colidx);
    cudaFree(g->vals);
    cudaFree(g->perm);
    if (g->st) cudaStreamDestroy(g->st);
}

}  // namespace

extern "C" {

int mr_graph_create(int32_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx, const void* vals,
                    int32_t dtype, int32_t graph_id, mr_graph** out)
{
    if (!out || n < 0 || nnz < 0 || nnz > INT32_MAX || !rowptr || (nnz > 0 && (!colidx || !vals)))
        return MR_ERR_INVALID_ARG;
    if (dtype != MR_F32 && dtype != MR_F16 && dtype != MR_BF16) return MR_ERR_UNSUPPORTED;
    *out = nullptr;
    auto* g = new (std::nothrow) mr_graph;
    if (!g) return MR_ERR_NOMEM;
    g->n = n;
    g->nnz = nnz;
    g->dtype = dtype;
    g->graph_id = graph_id;
    const size_t vb = dtype_size(dtype);
    if (cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&g->rowptr, sizeof(int32_t) * ((size_t)n + 1)) != cudaSuccess ||
        cudaMalloc(&g->colidx, sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1)) != cudaSuccess ||
        cudaMalloc(&g->vals, vb * (size_t)std::max<int64_t>(nnz, 1)) != cudaSuccess ||
        cudaMalloc(&g->perm, sizeof(int32_t) * (size_t)std::max(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        free_graph(g);
        delete g;
        return MR_ERR_NOMEM;
    }
    cudaMemcpyAsync(g->rowptr, rowptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, g->st);
    if (nnz > 0) {
        cudaMemcpyAsync(g->colidx, colidx, sizeof(int32_t) * (size_t)nnz, cudaMemcpyHostToDevice, g->st);
        cudaMemcpyAsync(g->vals, vals, vb * (size_t)nnz, cudaMemcpyHostToDevice, g->st);
    }
    if (n > 0) iota_kernel<<<grid_n(n), 256, 0, g->st>>>(g->perm, n);
    int ok = 0;
    const mr_csr_view v = g->view();
    int s = validate_csr(v, &ok, g->st);
    if (s != MR_OK || !ok) {
        free_graph(g);
        delete g;
        return s != MR_OK ? s : MR_ERR_INVALID_ARG;
    }
    *out = g;
    return MR_OK;
}

int mr_graph_destroy(mr_graph* g)
{
    if (!g) return MR_OK;
    cudaStreamSynchronize(g->st);
    free_graph(g);
    delete g;
    return MR_OK;
}

int mr_graph_gorder4(mr_graph* g, int32_t vsize, int32_t width, double* ms_order, double* ms_relabel)
{
    if (!g || width < 1) return MR_ERR_INVALID_ARG;
    const int32_t n = g->n;
    if (n == 0) return MR_OK;
    // the ordering: on the GPU when its queue fits (the same permutation),
    // else on host threads from host copies of the current structure (the
    // reference's D2H, src/class.cu:2642-2645)
    auto t0 = std::chrono::steady_clock::now();
    DevBuf step, n2o_dev;
    MR_TRY(step.alloc(sizeof(int32_t) * (size_t)n, g->st));
    MR_TRY(n2o_dev.alloc(sizeof(uint32_t) * (size_t)n, g->st));
    int rc = pgorder_gpu(n, g->rowptr, g->colidx, (int32_t)g->nnz, vsize, width, n2o_dev.as<uint32_t>(), g->st);
    if (rc == MR_OK) {
        MR_TRY(mr_perm_invert(n, reinterpret_cast<const int32_t*>(n2o_dev.p), step.as<int32_t>(), g->st));
    } else if (rc == MR_ERR_UNSUPPORTED) {
        std::vector<int32_t> hr((size_t)n + 1), hc((size_t)std::max<int64_t>(g->nnz, 1));
        MR_CUDA_TRY(cudaMemcpyAsync(hr.data(), g->rowptr, sizeof(int32_t) * hr.size(), cudaMemcpyDeviceToHost, g->st));
        MR_CUDA_TRY(
            cudaMemcpyAsync(hc.data(), g->colidx, sizeof(int32_t) * (size_t)g->nnz, cudaMemcpyDeviceToHost, g->st));
        MR_CUDA_TRY(cudaStreamSynchronize(g->st));
        t0 = std::chrono::steady_clock::now();
        std::vector<uint32_t> new2old((size_t)n);
        MR_TRY(pgorder_host(n, hr.data(), hc.data(), vsize, width, 0, new2old.data()));
        std::vector<int32_t> old2new((size_t)n);
        for (int32_t i = 0; i < n; ++i) old2new[new2old[(size_t)i]] = i;
        MR_CUDA_TRY(
            cudaMemcpyAsync(step.p, old2new.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, g->st));
        MR_CUDA_TRY(cudaStreamSynchronize(g->st));  // old2new is a host local
    } else {
        return rc;
    }
    if (ms_order) *ms_order = ms_since(t0);

    t0 = std::chrono::steady_clock::now();
    int32_t *nr = nullptr, *nc = nullptr;
    void* nv = nullptr;
    const size_t vb = dtype_size(g->dtype);
    if (cudaMalloc(&nr, sizeof(int32_t) * ((size_t)n + 1)) != cudaSuccess ||
        cudaMalloc(&nc, sizeof(int32_t) * (size_t)std::max<int64_t>(g->nnz, 1)) != cudaSuccess ||
        cudaMalloc(&nv, vb * (size_t)std::max<int64_t>(g->nnz, 1)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(nr);
        cudaFree(nc);
        cudaFree(nv);
        return MR_ERR_NOMEM;
    }
    const mr_csr_view v = g->view();
    int s = permute_csr(v, step.as<int32_t>(), nr, nc, nv, g->st);
    if (s != MR_OK) {
        cudaFree(nr);
        cudaFree(nc);
        cudaFree(nv);
        return s;
    }
    compose_kernel<<<grid_n(n), 256, 0, g->st>>>(step.as<int32_t>(), g->perm, n);
    MR_CUDA_TRY(cudaStreamSynchronize(g->st));
    cudaFree(g->rowptr);
    cudaFree(g->colidx);
    cudaFree(g->vals);
    g->rowptr = nr;
    g->colidx = nc;
    g->vals = nv;
    if (ms_relabel) *ms_relabel = ms_since(t0);
    return MR_OK;
}

int mr_graph_locality_predict(mr_graph* g, double* features10, float* speedup)
{
    if (!g) return MR_ERR_INVALID_ARG;
    return mr_locality_predict(g->colidx, (int32_t)g->nnz, g->n, g->graph_id, features10, speedup, g->st);
}

int mr_graph_gated_reorder(mr_graph* g, int32_t model, double tau_l, double tau_h, int32_t relabel_uncertain,
                           int32_t vsize, int32_t width, int32_t* decision, double* predicted)
{
    if (!g || width < 1) return MR_ERR_INVALID_ARG;
    double sp = 0.0;
    MR_TRY(mr_predict_reorder(g->colidx, (int32_t)g->nnz, g->n, g->graph_id, model, nullptr, &sp, g->st));
    int32_t d = MR_GATE_UNCERTAIN;
    MR_TRY(mr_band_gate(sp, tau_l, tau_h, &d));
    if (predicted) *predicted = sp;
    if (decision) *decision = d;
    if (d == MR_GATE_RELABEL || (d == MR_GATE_UNCERTAIN && relabel_uncertain))
        MR_TRY(mr_graph_gorder4(g, vsize, width, nullptr, nullptr));
    return MR_OK;
}

int mr_graph_spmv(mr_graph* g, const char* method, int32_t iters, const float* x_host, float* y_host,
                  double* ms_plan, double* ms_spmv)
{
    if (!g || !method || !y_host || iters < 1) return MR_ERR_INVALID_ARG;
    const std::string m(method);
    if (m != "csr" && m != "merbit") return MR_ERR_INVALID_ARG;
    const int32_t n = g->n;
    if (n == 0) return MR_OK;
    DevBuf x, xp, yp, y;
    MR_TRY(x.alloc(sizeof(float) * n, g->st));
    MR_TRY(xp.alloc(sizeof(float) * n, g->st));
    MR_TRY(yp.alloc(sizeof(float) * n, g->st));
    MR_TRY(y.alloc(sizeof(float) * n, g->st));
    if (x_host)
        MR_CUDA_TRY(cudaMemcpyAsync(x.p, x_host, sizeof(float) * n, cudaMemcpyHostToDevice, g->st));
    else
        fill_kernel<<<grid_n(n), 256, 0, g->st>>>(x.as<float>(), n, 1.0f);  // x = 1 (src/class.cu:1351-1353)
    MR_TRY(launch_permute_vector(n, g->perm, x.as<float>(), xp.as<float>(), 0, g->st));
    const mr_csr_view v = g->view();
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    mr_merbit_plan* plan = nullptr;
    int s = MR_OK;
    cudaEventRecord(e0, g->st);
    // SIGMA 14 as the reference (src/class.cu:1409-1410); the B200 kernel picks its own CTA shape
    if (m == "merbit") s = mr_merbit_plan_create(&v, 14, 0, g->st, &plan);
    cudaEventRecord(e1, g->st);
    for (int it = 0; it < iters && s == MR_OK; ++it)
        s = plan ? mr_spmv_merbit(plan, &v, xp.as<float>(), yp.as<float>(), g->st)
                 : mr_spmv_csr(&v, xp.as<float>(), yp.as<float>(), g->st);
    cudaEventRecord(e2, g->st);
    if (s == MR_OK) s = launch_permute_vector(n, g->perm, yp.as<float>(), y.as<float>(), 1, g->st);
    if (s == MR_OK && cudaMemcpyAsync(y_host, y.p, sizeof(float) * n, cudaMemcpyDeviceToHost, g->st) != cudaSuccess)
        s = MR_ERR_CUDA;
    if (cudaStreamSynchronize(g->st) != cudaSuccess) s = MR_ERR_CUDA;
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    if (ms_plan) *ms_plan = a;
    if (ms_spmv) *ms_spmv = b / iters;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (plan) mr_merbit_plan_destroy(plan);
    return s;
}

int mr_graph_get_perm(const mr_graph* g, int32_t* perm_host)
{
    if (!g || !perm_host) return MR_ERR_INVALID_ARG;
    if (g->n == 0) return MR_OK;
    MR_CUDA_TRY(cudaMemcpyAsync(perm_host, g->perm, sizeof(int32_t) * g->n, cudaMemcpyDeviceToHost, g->st));
    MR_CUDA_TRY(cudaStreamSynchronize(g->st));
    return MR_OK;
}

int mr_graph_view(const mr_graph* g, mr_csr_view* v)
{
    if (!g || !v) return MR_ERR_INVALID_ARG;
    *v = g->view();
    return MR_OK;
}

}  // extern "C"
