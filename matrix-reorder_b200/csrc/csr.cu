// Plain CSR SpMV for sm_100a (the reference's cuSPARSE CSR_ALG1 path,
// src/class.cu:1359-1397, replaced by a hand-written kernel).
//
// Two kernels, both deterministic (every row is summed by one lane group or
// one CTA, in a fixed order):
//  * csr_vector_kernel: groups of G lanes (G = 2..32, picked from the mean
//    row length), one row per group at a time; lanes stride the row with
//    evict-first loads of colidx and values, gather x through L2 with an
//    evict-last policy, and reduce with a fixed shuffle tree. Every warp owns
//    a contiguous chunk of rows and its groups take adjacent rows of the
//    chunk, so the loads of a warp stay coalesced and a heavy row lands in
//    its own warp: a plain grid-stride over rows would hand the rows that are
//    equal modulo the stride to the same group, and orders that start every
//    block of ids with its heaviest vertex (pGOrder partitions of 1024)
//    would then pile the heavy rows onto a few groups. With narrow groups
//    (MED), rows of more than kMedRow nonzeros are deferred to a per-warp
//    list in shared memory and summed afterwards by the whole warp; rows
//    longer than kLongRow are skipped and appended to a global list.
//  * csr_long_rows_kernel: one 1024-thread CTA per listed row, a fixed
//    per-thread stride (four loads in flight) and a fixed shared-memory tree.
#include "common.cuh"
#include "internal.hpp"

namespace mr {

constexpr int kLongRow = 4096;
constexpr int kLongThreads = 1024;
constexpr int kMedRow = 32;     // narrow groups defer longer rows to the whole warp
constexpr int kMedList = 256;   // deferral only for warps whose chunk has at most this many rows

template <typename V, int G, bool MED>
__global__ void __launch_bounds__(256)
    csr_vector_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx, const V* __restrict__ vals,
                      const float* __restrict__ x, float* __restrict__ y, int* __restrict__ long_rows,
                      int* __restrict__ n_long)
{
    constexpr int GPW = 32 / G;  // groups per warp
    __shared__ int s_med[MED ? 8 : 1][MED ? kMedList : 1];
    __shared__ int s_nmed[8];
    const uint64_t pol = l2_evict_last_policy();
    const int lane = threadIdx.x & (G - 1);
    const int gi = (threadIdx.x & 31) / G;
    // the group's own lanes: groups of one warp run different rows, so every
    // shuffle names only its group
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int chunk = ((n + warps - 1) / warps + GPW - 1) / GPW * GPW;
    const int r0 = min(n, warp * chunk), r1 = min(n, r0 + chunk);
    const int wl = (threadIdx.x >> 5);  // warp in the CTA
    // deferring only when the whole chunk fits the list keeps the choice of
    // who sums a row independent of timing
    const bool defer = MED && (r1 - r0) <= kMedList;
    if (MED && (threadIdx.x & 31) == 0) s_nmed[wl] = 0;
    __syncwarp();
    for (int row = r0 + gi; row < r1; row += GPW) {
        const int b = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
        if (e - b > kLongRow) {
            if (lane == 0) long_rows[atomicAdd(n_long, 1)] = row;
            continue;
        }
        if constexpr (MED) {
            if (defer && e - b > kMedRow) {
                if (lane == 0) s_med[wl][atomicAdd(&s_nmed[wl], 1)] = row;
                continue;  // the warp sums it below
            }
        }
        float s = 0.f;
        for (int k = b + lane; k < e; k += G)
            s += ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol);
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(gmask, s, o, G);
        if (lane == 0) y[row] = s;
    }
    if constexpr (MED) {
        // deferred rows, in list order, one warp each
        __syncwarp();
        const int l = threadIdx.x & 31;
        const int cnt = s_nmed[wl];
        for (int i = 0; i < cnt; ++i) {
            const int row = s_med[wl][i];
            const int b = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
            float s = 0.f;
            for (int k = b + l; k < e; k += 32)
                s += ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol);
            s = warp_sum(s);
            if (l == 0) y[row] = s;
        }
    }
}

template <typename V>
__global__ void __launch_bounds__(kLongThreads)
    csr_long_rows_kernel(const int* __restrict__ rowptr, const int* __restrict__ colidx, const V* __restrict__ vals,
                         const float* __restrict__ x, float* __restrict__ y, const int* __restrict__ long_rows,
                         const int* __restrict__ n_long)
{
    __shared__ float s_part[kLongThreads / 32];
    const uint64_t pol = l2_evict_last_policy();
    const int count = *n_long;
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const int row = long_rows[i];
        const int b = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        int k = b + (int)threadIdx.x;
        for (; k + 3 * kLongThreads < e; k += 4 * kLongThreads) {
            s0 += ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol);
            s1 += ValueTraits<V>::f(ld_stream(vals + k + kLongThreads)) *
                  ld_x(x + ld_stream(colidx + k + kLongThreads), pol);
            s2 += ValueTraits<V>::f(ld_stream(vals + k + 2 * kLongThreads)) *
                  ld_x(x + ld_stream(colidx + k + 2 * kLongThreads), pol);
            s3 += ValueTraits<V>::f(ld_stream(vals + k + 3 * kLongThreads)) *
                  ld_x(x + ld_stream(colidx + k + 3 * kLongThreads), pol);
        }
        for (; k < e; k += kLongThreads)
            s0 += ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol);
        float s = (s0 + s1) + (s2 + s3);
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            float t = s_part[threadIdx.x];
            t = warp_sum(t);
            if (threadIdx.x == 0) y[row] = t;
        }
        __syncthreads();
    }
}

template <typename V>
static int launch_t(int n, int64_t nnz, const int* rowptr, const int* colidx, const void* vals, const float* x, float* y,
                    cudaStream_t st)
{
    DevBuf list;
    const int64_t max_long = nnz / (kLongRow + 1) + 1;
    MR_TRY(list.alloc(sizeof(int) * (size_t)(max_long + 1), st));
    int* n_long = list.as<int>();
    int* long_rows = n_long + 1;
    MR_CUDA_TRY(cudaMemsetAsync(n_long, 0, sizeof(int), st));
    const V* v = reinterpret_cast<const V*>(vals);
    // lanes per row from the mean row length; below 24 the groups stay narrow
    // and rows above kMedRow go to the whole warp
    const double mean = (double)nnz / (double)n;
    const int g = mean <= 3 ? 2 : mean <= 6 ? 4 : mean <= 24 ? 8 : 32;
    const long long want = ((long long)n * g + 255) / 256;
    const int grid = (int)std::max<long long>(1, std::min<long long>(want, (long long)sm_count() * 32));
    switch (g) {
    case 2: csr_vector_kernel<V, 2, true><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y, long_rows, n_long); break;
    case 4: csr_vector_kernel<V, 4, true><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y, long_rows, n_long); break;
    case 8: csr_vector_kernel<V, 8, true><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y, long_rows, n_long); break;
    default:
        csr_vector_kernel<V, 32, false><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y, long_rows, n_long);
        break;
    }
    MR_CUDA_TRY(cudaGetLastError());
    if (nnz > kLongRow) {
        const int lg = (int)std::max<int64_t>(1, std::min<int64_t>(max_long, (int64_t)sm_count() * 2));
        csr_long_rows_kernel<V><<<lg, kLongThreads, 0, st>>>(rowptr, colidx, v, x, y, long_rows, n_long);
        MR_CUDA_TRY(cudaGetLastError());
    }
    return MR_OK;
}

int launch_csr_spmv(int n, int64_t nnz, const int* rowptr, const int* colidx, const void* vals, int dtype,
                    const float* x, float* y, cudaStream_t st)
{
    if (n == 0) return MR_OK;
    switch (dtype) {
    case MR_F32: return launch_t<float>(n, nnz, rowptr, colidx, vals, x, y, st);
    case MR_F16: return launch_t<__half>(n, nnz, rowptr, colidx, vals, x, y, st);
    case MR_BF16: return launch_t<__nv_bfloat16>(n, nnz, rowptr, colidx, vals, x, y, st);
    default: return MR_ERR_UNSUPPORTED;
    }
}

}  // namespace mr
