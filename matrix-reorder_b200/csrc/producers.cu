// Simple permutation producers on the GPU, the reference's comparators for
// pGOrder: degree order, DBG (degree-based grouping) and a seeded random
// order. Each returns perm[old] = new for mr_permute_csr.
//
//  * degree (GRAPH::relabel_degree, src/class.cu:1493-1549): vertices by
//    decreasing degree, ties by increasing id. The degree of v is the number
//    of nonzeros in column v (the reference counts its row_ind array, which
//    holds our column indices, desc_kernel1 at src/class.cu:473-481); its
//    descending sort_by_key on integer keys is a stable radix sort, hence
//    the id tie-break.
//  * DBG (GRAPH::dbg, src/class.cu:1660-1760): the same degree, grouped by
//    class ceilf(log2(deg + 1.0)) (dbg_kernel, src/class.cu:1682-1690),
//    classes in decreasing order, ids increasing inside a class
//    (DegIdCompare, src/class.cu:1673-1679).
//  * random (GRAPH::relabel_random, src/class.cu:1460-1491): a seeded
//    uniform permutation. The reference uses thrust::shuffle with
//    thrust::default_random_engine(graph_id); this is our own shuffle
//    (a 32-bit hash of (seed, id) as the sort key, ties by id), not the same
//    permutation as the reference's for the same seed.
//
// All three are one counting kernel (degree producers), one key kernel, a
// stable LSD radix sort of (key, id) and one scatter perm[id] = rank.
#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

__global__ void column_count_kernel(const int32_t* __restrict__ colidx, int64_t nnz, int ncols, uint32_t* __restrict__ cnt,
                                    int* __restrict__ bad)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int c = colidx[k];
        if (c < 0 || c >= ncols)
            atomicOr(bad, 1);
        else
            atomicAdd(&cnt[c], 1u);
    }
}

// key = ~degree (ascending key = descending degree) or 255 - DBG class
__global__ void degree_key_kernel(uint32_t* __restrict__ key, int32_t* __restrict__ id, int n, int dbg)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t d = key[v];
        if (dbg) {
            // the reference's expression: double log2, then ceilf of its float value
            const int cls = (int)ceilf(log2((double)d + 1.0));
            key[v] = 255u - (uint32_t)cls;
        } else {
            key[v] = ~d;
        }
        id[v] = v;
    }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    // murmur3 finaliser
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

__global__ void random_key_kernel(uint32_t* __restrict__ key, int32_t* __restrict__ id, int n, uint32_t seed)
{
    const uint32_t s = mix32(seed ^ 0x9e3779b9u);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        key[v] = mix32((uint32_t)v * 0x27d4eb2fu + s);
        id[v] = v;
    }
}

__global__ void rank_scatter_kernel(const int32_t* __restrict__ id, int n, int32_t* __restrict__ perm)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) perm[id[k]] = k;
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8)); }

// kind: 0 degree, 1 DBG, 2 random
int produce(const mr_csr_view* A, int n, int kind, uint32_t seed, int32_t* perm, cudaStream_t st)
{
    if (n == 0) return MR_OK;
    DevBuf k0, k1, v0, v1, flag;
    MR_TRY(k0.alloc(sizeof(uint32_t) * (size_t)n, st));
    MR_TRY(k1.alloc(sizeof(uint32_t) * (size_t)n, st));
    MR_TRY(v0.alloc(sizeof(int32_t) * (size_t)n, st));
    MR_TRY(v1.alloc(sizeof(int32_t) * (size_t)n, st));
    int bits = 32;
    if (kind == 2) {
        random_key_kernel<<<grid_n(n), 256, 0, st>>>(k0.as<uint32_t>(), v0.as<int32_t>(), n, seed);
    } else {
        MR_TRY(flag.alloc(sizeof(int), st));
        MR_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        MR_CUDA_TRY(cudaMemsetAsync(k0.p, 0, sizeof(uint32_t) * (size_t)n, st));
        if (A->nnz > 0)
            column_count_kernel<<<grid_n(A->nnz), 256, 0, st>>>(A->colidx, A->nnz, n, k0.as<uint32_t>(), flag.as<int>());
        degree_key_kernel<<<grid_n(n), 256, 0, st>>>(k0.as<uint32_t>(), v0.as<int32_t>(), n, kind == 1);
        int h = 0;
        MR_CUDA_TRY(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MR_CUDA_TRY(cudaStreamSynchronize(st));
        if (h) return MR_ERR_INVALID_ARG;
        if (kind == 1) bits = 8;
    }
    MR_CUDA_TRY(cudaGetLastError());
    uint32_t* keys = k0.as<uint32_t>();
    int32_t* ids = v0.as<int32_t>();
    MR_TRY(radix_sort_pairs_u32(keys, ids, k1.as<uint32_t>(), v1.as<int32_t>(), n, bits, st));
    rank_scatter_kernel<<<grid_n(n), 256, 0, st>>>(ids, n, perm);
    MR_CUDA_TRY(cudaGetLastError());
    MR_CUDA_TRY(cudaStreamSynchronize(st));  // the sort's buffers are released on return
    return MR_OK;
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" {

int mr_order_degree(const mr_csr_view* A, int32_t* perm_old2new, void* stream)
{
    if (!A || !perm_old2new || A->n_rows != A->n_cols || A->n_rows < 0 || A->nnz < 0 || (A->nnz > 0 && !A->colidx))
        return MR_ERR_INVALID_ARG;
    return produce(A, A->n_rows, 0, 0, perm_old2new, as_stream(stream));
}

int mr_order_dbg(const mr_csr_view* A, int32_t* perm_old2new, void* stream)
{
    if (!A || !perm_old2new || A->n_rows != A->n_cols || A->n_rows < 0 || A->nnz < 0 || (A->nnz > 0 && !A->colidx))
        return MR_ERR_INVALID_ARG;
    return produce(A, A->n_rows, 1, 0, perm_old2new, as_stream(stream));
}

int mr_order_random(int32_t n, uint32_t seed, int32_t* perm_old2new, void* stream)
{
    if (n < 0 || (n > 0 && !perm_old2new)) return MR_ERR_INVALID_ARG;
    return produce(nullptr, n, 2, seed, perm_old2new, as_stream(stream));
}

}  // extern "C"
