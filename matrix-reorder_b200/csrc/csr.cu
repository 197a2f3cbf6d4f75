// Plain CSR SpMV for sm_100a (the reference's cuSPARSE CSR_ALG1 path,
// src/class.cu:1359-1397, replaced by a hand-written kernel).
//
// A group of G lanes (G = 4..32, picked from the mean row length) owns one
// row at a time; lanes stride the row with evict-first loads of colidx and
// values, gather x through L2 with an evict-last policy, and reduce with a
// fixed shuffle tree, so the result is deterministic.
#include "common.cuh"
#include "internal.hpp"

namespace mr {

template <typename V, int G>
__global__ void __launch_bounds__(256)
    csr_vector_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx, const V* __restrict__ vals,
                      const float* __restrict__ x, float* __restrict__ y)
{
    const uint64_t pol = l2_evict_last_policy();
    const int lane = threadIdx.x & (G - 1);
    const int groups = (gridDim.x * blockDim.x) / G;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < n; row += groups) {
        const int b = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
        float s = 0.f;
        for (int k = b + lane; k < e; k += G)
            s += ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol);
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
        if (lane == 0) y[row] = s;
    }
}

template <typename V>
static void launch_g(int g, int n, const int* rowptr, const int* colidx, const void* vals, const float* x, float* y,
                     cudaStream_t st)
{
    const long long want = ((long long)n * g + 255) / 256;
    const int grid = (int)std::min<long long>(want, (long long)sm_count() * 32);
    const V* v = reinterpret_cast<const V*>(vals);
    switch (g) {
    case 2: csr_vector_kernel<V, 2><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y); break;
    case 4: csr_vector_kernel<V, 4><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y); break;
    case 8: csr_vector_kernel<V, 8><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y); break;
    case 16: csr_vector_kernel<V, 16><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y); break;
    default: csr_vector_kernel<V, 32><<<grid, 256, 0, st>>>(n, rowptr, colidx, v, x, y); break;
    }
}

int launch_csr_spmv(int n, int64_t nnz, const int* rowptr, const int* colidx, const void* vals, int dtype,
                    const float* x, float* y, cudaStream_t st)
{
    if (n == 0) return MR_OK;
    const double mean = (double)nnz / (double)n;
    const int g = mean <= 3 ? 2 : mean <= 6 ? 4 : mean <= 12 ? 8 : mean <= 24 ? 16 : 32;
    switch (dtype) {
    case MR_F32: launch_g<float>(g, n, rowptr, colidx, vals, x, y, st); break;
    case MR_F16: launch_g<__half>(g, n, rowptr, colidx, vals, x, y, st); break;
    case MR_BF16: launch_g<__nv_bfloat16>(g, n, rowptr, colidx, vals, x, y, st); break;
    default: return MR_ERR_UNSUPPORTED;
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

}  // namespace mr
