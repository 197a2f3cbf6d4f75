// Gather-ceiling probe: the bandwidth a B200 reaches on the x-gather part of
// SpMV alone, for a given column-index stream.
//
// The kernel streams colidx and values with 16-byte evict-first loads and
// gathers x[colidx[k]] (read-only path, L2 evict-last), summing the products
// without any row structure, descriptor, scan or y write. Its time is a lower
// bound for any CSR-style SpMV that needs one x gather per nonzero on the
// same stream, which is why SpMV time is reported against it next to the HBM
// roofline.
#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

__global__ void __launch_bounds__(1024) gather_probe_kernel(const int4* __restrict__ idx, const float4* __restrict__ val,
                                                            long long n4, const float* __restrict__ x,
                                                            float* __restrict__ sink)
{
    const uint64_t pol = l2_evict_last_policy();
    float s = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const int4 c = ld_stream(idx + i);
        const float4 v = ld_stream(val + i);
        s += v.x * ld_x(x + c.x, pol) + v.y * ld_x(x + c.y, pol) + v.z * ld_x(x + c.z, pol) + v.w * ld_x(x + c.w, pol);
    }
    if (s == 1.2345e-30f) sink[0] = s;  // keeps the loads alive
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" int mr_gather_ceiling(const int32_t* colidx, const float* vals, int64_t nnz, const float* x, int32_t reps,
                                 float* ms_per_pass, void* stream)
{
    if (!colidx || !vals || !x || !ms_per_pass || nnz < 4 || reps < 1) return MR_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(colidx) & 15) || (reinterpret_cast<uintptr_t>(vals) & 15))
        return MR_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    DevBuf sink;
    MR_TRY(sink.alloc(sizeof(float), st));
    const long long n4 = nnz / 4;  // the last nnz % 4 entries are left out
    const int grid = sm_count() * 2;
    cudaEvent_t a, b;
    MR_CUDA_TRY(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return MR_ERR_CUDA;
    }
    for (int w = 0; w < 2; ++w)
        gather_probe_kernel<<<grid, 1024, 0, st>>>(reinterpret_cast<const int4*>(colidx),
                                                   reinterpret_cast<const float4*>(vals), n4, x, sink.as<float>());
    cudaEventRecord(a, st);
    for (int r = 0; r < reps; ++r)
        gather_probe_kernel<<<grid, 1024, 0, st>>>(reinterpret_cast<const int4*>(colidx),
                                                   reinterpret_cast<const float4*>(vals), n4, x, sink.as<float>());
    cudaEventRecord(b, st);
    const cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    MR_CUDA_TRY(e);
    MR_CUDA_TRY(cudaGetLastError());
    *ms_per_pass = ms / reps;
    return MR_OK;
}
