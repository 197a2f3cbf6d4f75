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
//  * random (GRAPH::relabel_random, src/class.cu:1460-1491): the same
//    permutation as the reference's thrust::shuffle of the identity with
//    thrust::default_random_engine seeded with graph_id, bit for bit (the
//    Feistel bijection below).
//
// Degree and DBG are one counting kernel, one key kernel, a stable LSD radix
// sort of (key, id) and one scatter perm[id] = rank; random is a flag pass,
// a scan and a scatter over the bijection's domain.
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

// ---- random order: the permutation of thrust::shuffle --------------------
// GRAPH::relabel_random shuffles the identity perm with thrust::shuffle and
// thrust::default_random_engine seeded with graph_id (src/class.cu:1467-1473).
// Thrust's shuffle (thrust/system/detail/generic/shuffle.inl, CCCL of CUDA
// 12.9) draws 24 round keys from the engine, maps every index of
// [0, 2^bits) through a 24-round Feistel network (bits = 4 up to 16
// elements, else ceil(log2 n)) and keeps, in index order, the images that
// fall below n: out[j] = image of the j-th such index. The round function
// and its multiplier must be Thrust's for the same permutation; the
// compaction here is a flag pass, a device scan and a scatter.
struct FeistelKeys {
    uint32_t key[24];
    uint32_t lbits, rbits;
};

FeistelKeys feistel_keys(int n, uint32_t seed)
{
    // minstd_rand: x <- 48271 x mod (2^31 - 1); a zero seed becomes 1
    uint64_t x = seed % 2147483647u;
    if (x == 0) x = 1;
    FeistelKeys f;
    for (int i = 0; i < 24; ++i) {
        x = x * 48271u % 2147483647u;
        f.key[i] = (uint32_t)x;
    }
    uint32_t bits = 4;
    if (n > 16) {
        bits = 0;
        for (uint32_t m = (uint32_t)n - 1; m; m >>= 1) ++bits;
    }
    f.lbits = bits / 2;
    f.rbits = bits - f.lbits;
    return f;
}

__device__ __forceinline__ uint32_t feistel_image(const FeistelKeys& f, uint32_t v)
{
    const uint32_t lmask = (1u << f.lbits) - 1u, rmask = (1u << f.rbits) - 1u;
    uint32_t a = v >> f.rbits, b = v & rmask;
#pragma unroll
    for (int r = 0; r < 24; ++r) {
        const uint64_t p = 0xD2B74407B1CE6E93ull * (uint64_t)a;
        const uint32_t lo = ((uint32_t)p << (f.rbits - f.lbits)) | (b >> f.lbits);
        a = ((uint32_t)(p >> 32) ^ f.key[r] ^ b) & lmask;
        b = lo & rmask;
    }
    return (a << f.rbits) | b;
}

__global__ void shuffle_flag_kernel(const FeistelKeys f, int64_t span, int n, int32_t* __restrict__ flag)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < span; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = feistel_image(f, (uint32_t)v) < (uint32_t)n ? 1 : 0;
}

__global__ void shuffle_scatter_kernel(const FeistelKeys f, int64_t span, int n, const int32_t* __restrict__ pos,
                                       int32_t* __restrict__ perm)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < span; v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = feistel_image(f, (uint32_t)v);
        if (k < (uint32_t)n) perm[pos[v]] = (int32_t)k;
    }
}

__global__ void rank_scatter_kernel(const int32_t* __restrict__ id, int n, int32_t* __restrict__ perm)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) perm[id[k]] = k;
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8)); }

// kind: 0 degree, 1 DBG, 2 random
int shuffle_order(int n, uint32_t seed, int32_t* perm, cudaStream_t st)
{
    const FeistelKeys f = feistel_keys(n, seed);
    const int64_t span = 1ll << (f.lbits + f.rbits);
    DevBuf flag, pos;
    MR_TRY(flag.alloc(sizeof(int32_t) * (size_t)span, st));
    MR_TRY(pos.alloc(sizeof(int32_t) * ((size_t)span + 1), st));
    shuffle_flag_kernel<<<grid_n(span), 256, 0, st>>>(f, span, n, flag.as<int32_t>());
    MR_CUDA_TRY(cudaGetLastError());
    MR_TRY(exclusive_scan_i32(flag.as<int32_t>(), pos.as<int32_t>(), span, st));
    shuffle_scatter_kernel<<<grid_n(span), 256, 0, st>>>(f, span, n, pos.as<int32_t>(), perm);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;  // the pool keeps flag / pos ordered on st
}

int produce(const mr_csr_view* A, int n, int kind, uint32_t seed, int32_t* perm, cudaStream_t st)
{
    if (n == 0) return MR_OK;
    if (kind == 2) return shuffle_order(n, seed, perm, st);
    DevBuf k0, k1, v0, v1, flag;
    MR_TRY(k0.alloc(sizeof(uint32_t) * (size_t)n, st));
    MR_TRY(k1.alloc(sizeof(uint32_t) * (size_t)n, st));
    MR_TRY(v0.alloc(sizeof(int32_t) * (size_t)n, st));
    MR_TRY(v1.alloc(sizeof(int32_t) * (size_t)n, st));
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
    const int bits = kind == 1 ? 8 : 32;
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
