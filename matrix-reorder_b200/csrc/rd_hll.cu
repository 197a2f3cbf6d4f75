// Sampled reuse distance with HyperLogLog registers on sm_100a.
//
// Semantics are the reference's sampled_hll_rd_block_kernel
// (src/class.cu:1014-1131) and its host binning (:1213-1256): sample sid sits
// at pos = 1 + hash(seed ^ (sid*0x9e3779b9 + 17)) % (nnz-1); the stream is
// scanned backwards from pos-1 in 256-position chunks; every sector other
// than the target's is inserted into 2^p registers (max of ranks) until the
// chunk holding the previous occurrence of the target sector, of which only
// the positions above that occurrence count; every 16 chunks without a hit
// the estimate is compared against 1.03 * rd_cap. Status 0 found, 1 cold,
// 2 capped, 3 max_scan reached.
//
// B200 restatement (same registers, statuses and estimates, bit for bit):
//  * one CTA of 512 threads per sample scans a whole 16-chunk group (4096
//    positions, 8 coalesced loads per thread) per step with 3 barriers,
//    where the reference pays 3 barriers per 256 positions. Registers are a
//    max, so the insertion order inside a group does not matter, and the
//    only cap check the reference can make inside a group is at its end.
//  * the cap check uses the exact register sum (fixed point, 64-bit integer
//    block reduction); only when that decision lies within 1e-3 of the
//    threshold, and for every estimate that is reported, is the reference's
//    sequential FP32 sum replayed in register order, so reported estimates
//    are the reference's floats exactly.
#include <algorithm>

#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

constexpr int kHllThreads = 512;
constexpr int kChunk = 256;          // reference chunk (its block size)
constexpr int kGroupChunks = 16;     // reference cap-check cadence
constexpr int kGroup = kChunk * kGroupChunks;
constexpr int kPerThread = kGroup / kHllThreads;

__host__ __device__ __forceinline__ uint32_t hll_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ int hll_rank(uint32_t h, int p)
{
    const uint32_t w = h >> p;
    const int max_rank = 32 - p + 1;
    if (w == 0U) return max_rank;
    int r = __clz(w) - p + 1;
    return min(max(r, 1), max_rank);
}

__device__ __forceinline__ float hll_alpha(int m)
{
    if (m == 16) return 0.673f;
    if (m == 32) return 0.697f;
    if (m == 64) return 0.709f;
    return 0.7213f / (1.0f + 1.079f / (float)m);
}

// The reference's estimate: FP32 sum of exp2f(-r) in register order. Terms
// are computed in parallel into `terms`, then thread 0 adds them in order.
__device__ float hll_estimate_replay(const int* regs, float* terms, int m, float* s_out)
{
    for (int i = threadIdx.x; i < m; i += blockDim.x) terms[i] = exp2f(-(float)regs[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
        float sum = 0.0f;
        int zeros = 0;
        for (int i = 0; i < m; i += 8) {
            float t[8];
            int z[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                t[j] = terms[i + j];
                z[j] = regs[i + j];
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (z[j] == 0) ++zeros;
                sum += t[j];
            }
        }
        const float mf = (float)m;
        const float alpha = hll_alpha(m);
        float e = alpha * mf * mf / sum;
        if (e <= 2.5f * mf && zeros > 0) e = mf * logf(mf / (float)zeros);
        *s_out = e;
    }
    __syncthreads();
    return *s_out;
}

struct Exact {
    double est_raw;
    int zeros;
};

// exact register sum: sum 2^-r as a 64-bit fixed-point integer (scale 2^32;
// ranks are <= 29 and at most 2^14 registers, so it cannot overflow)
__device__ Exact hll_exact(const int* regs, int m, long long* s_red, int* s_zero)
{
    long long s = 0;
    int z = 0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int r = regs[i];
        s += 1ll << (32 - r);
        z += (r == 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_red[w] = s;
        s_zero[w] = z;
    }
    __syncthreads();
    long long S = 0;
    int Z = 0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
        S += s_red[j];
        Z += s_zero[j];
    }
    __syncthreads();
    const double sum = (double)S / 4294967296.0;
    const double mf = (double)m;
    return {(double)hll_alpha(m) * mf * mf / sum, Z};
}

__global__ void __launch_bounds__(kHllThreads)
    hll_sample_kernel(const int32_t* __restrict__ stream, int nnz, int samples, int sector, uint32_t seed, int rd_cap,
                      int max_scan, int p, float* __restrict__ est_out, int32_t* __restrict__ status_out,
                      int32_t* __restrict__ pos_out, int* __restrict__ next_sample)
{
    extern __shared__ int smem[];
    const int m = 1 << p;
    int* regs = smem;
    float* terms = reinterpret_cast<float*>(smem + m);
    __shared__ int s_found;
    __shared__ float s_est;
    __shared__ long long s_red[kHllThreads / 32];
    __shared__ int s_zero[kHllThreads / 32];
    __shared__ int s_sid;

    // samples differ wildly in cost (a first touch scans the whole prefix):
    // hand them out dynamically
    for (;;) {
        if (threadIdx.x == 0) s_sid = atomicAdd(next_sample, 1);
        __syncthreads();
        const int sid = s_sid;
        if (sid >= samples) break;
        for (int i = threadIdx.x; i < m; i += kHllThreads) regs[i] = 0;
        const uint32_t r = hll_hash(seed ^ (uint32_t)((uint32_t)sid * 0x9e3779b9U + 17U));
        const int pos = 1 + (int)(r % (uint32_t)(nnz - 1));
        const int lo = (max_scan > 0) ? max(0, pos - max_scan) : 0;
        const int target = __ldg(stream + pos) / sector;
        const int total_chunks = (pos - 1 >= lo) ? (pos - 1 - lo) / kChunk + 1 : 0;
        const float thr = (float)rd_cap * 1.03f;
        int status = -99;
        float est = 0.0f;
        __syncthreads();
        for (int g = 0; g * kGroupChunks < total_chunks; ++g) {
            const int hi = pos - 1 - g * kGroup;
            if (threadIdx.x == 0) s_found = -1;
            int sec[kPerThread];
#pragma unroll
            for (int j = 0; j < kPerThread; ++j) {
                const int idx = hi - (int)threadIdx.x - j * kHllThreads;
                sec[j] = (idx >= lo) ? __ldg(stream + idx) / sector : -1;
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < kPerThread; ++j)
                if (sec[j] == target && sec[j] >= 0) atomicMax(&s_found, hi - (int)threadIdx.x - j * kHllThreads);
            __syncthreads();
            const int found = s_found;
#pragma unroll
            for (int j = 0; j < kPerThread; ++j) {
                const int idx = hi - (int)threadIdx.x - j * kHllThreads;
                if (idx >= lo && sec[j] != target && (found < 0 || idx > found)) {
                    const uint32_t h = hll_hash((uint32_t)sec[j]);
                    atomicMax(&regs[h & (uint32_t)(m - 1)], hll_rank(h, p));
                }
            }
            __syncthreads();
            if (found >= 0) {
                est = hll_estimate_replay(regs, terms, m, &s_est);
                status = 0;
                break;
            }
            const bool full_group = (g + 1) * kGroupChunks <= total_chunks;
            if (rd_cap > 0 && full_group) {
                const Exact ex = hll_exact(regs, m, s_red, s_zero);
                const double mf = (double)m;
                double e = ex.est_raw;
                const bool near_switch = fabs(e - 2.5 * mf) <= 1e-3 * 2.5 * mf;
                if (e <= 2.5 * mf && ex.zeros > 0) e = mf * log(mf / (double)ex.zeros);
                const bool near_thr = fabs(e - (double)thr) <= 1e-3 * (double)thr;
                bool exceed = e > (double)thr;
                float e_f = 0.0f;
                if (near_switch || near_thr || exceed) {
                    e_f = hll_estimate_replay(regs, terms, m, &s_est);
                    exceed = e_f > thr;
                }
                if (exceed) {
                    est = e_f;
                    status = 2;
                    break;
                }
            }
        }
        if (status == -99) {
            est = hll_estimate_replay(regs, terms, m, &s_est);
            status = (lo == 0) ? 1 : 3;
        }
        if (threadIdx.x == 0) {
            est_out[sid] = est;
            status_out[sid] = status;
            pos_out[sid] = pos;
        }
        __syncthreads();
    }
}

// host binning of src/class.cu:1213-1256, on the device
__global__ void hll_bin_kernel(const float* __restrict__ est, const int32_t* __restrict__ status, int samples,
                               const int32_t* __restrict__ edges, int nedges, unsigned long long* __restrict__ out)
{
    __shared__ unsigned long long h[64 + 4];
    for (int i = threadIdx.x; i < 68; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < samples; i += blockDim.x) {
        const int s = status[i];
        if (s == 0) {
            const double v = (double)est[i];
            int b = 0;
            while (b < nedges && (double)edges[b] <= v) ++b;
            atomicAdd(&h[b], 1ull);
            atomicAdd(&h[64 + 0], 1ull);
        } else if (s == 1) {
            atomicAdd(&h[64 + 1], 1ull);
        } else if (s == 2) {
            atomicAdd(&h[nedges], 1ull);
            atomicAdd(&h[64 + 2], 1ull);
        } else {
            atomicAdd(&h[64 + 3], 1ull);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= nedges; i += blockDim.x) out[i] = h[i];
    if (threadIdx.x < 4) out[nedges + 1 + threadIdx.x] = h[64 + threadIdx.x];
}

}  // namespace

int rd_hist_sampled(const int32_t* stream, int32_t nnz, int32_t samples, int32_t sector, int32_t rd_cap, int32_t hll_p,
                    int32_t max_scan, uint32_t seed, const int32_t* edges, int32_t nedges, int64_t* counts,
                    int64_t* stats, float* est, int32_t* status, int32_t* pos, cudaStream_t st)
{
    for (int b = 0; b <= nedges; ++b) counts[b] = 0;
    for (int b = 0; b < 4; ++b) stats[b] = 0;
    if (samples <= 0 || nnz <= 1) return MR_OK;
    int p = hll_p <= 0 ? 12 : hll_p;
    p = std::max(4, std::min(p, 14));
    const int m = 1 << p;
    const size_t smem = sizeof(int) * (size_t)m * 2;
    DevBuf b_est, b_status, b_pos, b_edges, b_out, b_next;
    if (!est) {
        MR_TRY(b_est.alloc(sizeof(float) * samples, st));
        est = b_est.as<float>();
    }
    if (!status) {
        MR_TRY(b_status.alloc(sizeof(int32_t) * samples, st));
        status = b_status.as<int32_t>();
    }
    if (!pos) {
        MR_TRY(b_pos.alloc(sizeof(int32_t) * samples, st));
        pos = b_pos.as<int32_t>();
    }
    MR_TRY(b_edges.alloc(sizeof(int32_t) * nedges, st));
    MR_TRY(b_out.alloc(sizeof(unsigned long long) * (nedges + 5), st));
    MR_TRY(b_next.alloc(sizeof(int), st));
    MR_CUDA_TRY(cudaMemsetAsync(b_next.p, 0, sizeof(int), st));
    MR_CUDA_TRY(cudaFuncSetAttribute(hll_sample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = std::min(samples, sm_count() * 4);
    hll_sample_kernel<<<grid, kHllThreads, smem, st>>>(stream, nnz, samples, sector, seed, rd_cap, max_scan, p, est,
                                                      status, pos, b_next.as<int>());
    MR_CUDA_TRY(cudaGetLastError());
    MR_CUDA_TRY(cudaMemcpyAsync(b_edges.p, edges, sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st));
    hll_bin_kernel<<<1, 1024, 0, st>>>(est, status, samples, b_edges.as<int32_t>(), nedges,
                                       b_out.as<unsigned long long>());
    MR_CUDA_TRY(cudaGetLastError());
    unsigned long long h[64 + 5];
    MR_CUDA_TRY(cudaMemcpyAsync(h, b_out.p, sizeof(unsigned long long) * (nedges + 5), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    for (int b = 0; b <= nedges; ++b) counts[b] = (int64_t)h[b];
    for (int b = 0; b < 4; ++b) stats[b] = (int64_t)h[nedges + 1 + b];
    return MR_OK;
}

}  // namespace mr

extern "C" uint32_t mr_hll_seed(int32_t graph_id, int32_t stream_type)
{
    // src/class.cu:1203
    return 246813579U + (uint32_t)graph_id * 1009U + (uint32_t)stream_type * 9176U;
}
