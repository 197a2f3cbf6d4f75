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
#include <atomic>
#include <climits>

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

#ifndef CSR_STREAM
#define CSR_STREAM 1
#endif
constexpr int kQ = 4;           // consecutive nonzeros per lane in a tile
constexpr int kTile = 32 * kQ;  // nonzeros per warp tile
constexpr int kTiles = 2;       // tiles whose loads are issued together

// Row of element k: the last row r in [rcur, rend) whose first nonzero is at
// or before k (an empty row shares its start with the next row, so this is
// the row that holds k; rowptr[rcur] <= k is required). *nxt receives
// rowptr[r + 1], the start of the rows after it (eb when r = rend - 1).
// Warp-wide: every lane calls it with its own k.
__device__ __forceinline__ int csr_row_of(const int* __restrict__ rowptr, int rcur, int rend, int eb, int k, int lane,
                                          int* nxt)
{
    int row = rcur, next = eb;
    bool more = true;
    for (int b = rcur + 1; b < rend; b += 32) {
        if (!__any_sync(0xffffffffu, more)) break;
        const int q = b + lane;
        const int sq = q < rend ? __ldg(rowptr + q) : INT_MAX;  // starts of rows b .. b+31 (sorted)
        int c = 0;                                              // how many of them are <= k
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
            const int sv = __shfl_sync(0xffffffffu, sq, c + st - 1);
            if (sv <= k) c += st;
        }
        const int s31 = __shfl_sync(0xffffffffu, sq, 31);
        if (c == 31 && s31 <= k) c = 32;
        const int sn = __shfl_sync(0xffffffffu, sq, c & 31);
        if (more) {
            row += c;
            if (c < 32) {
                next = sn == INT_MAX ? eb : sn;
                more = false;
            }
        }
    }
    *nxt = next;
    return row;
}

template <typename V, bool VEC>
__device__ __forceinline__ void csr_quad(const int* __restrict__ colidx, const V* __restrict__ vals,
                                         const float* __restrict__ x, uint64_t pol, int k0, int ea, int eb,
                                         float (&p)[kQ])
{
    if (VEC && k0 >= ea && k0 + kQ <= eb) {
        const int4 c = ld_stream(reinterpret_cast<const int4*>(colidx + k0));
        float v[4];
        Vec4<V>::unpack(ld_stream(reinterpret_cast<const typename Vec4<V>::T*>(vals + k0)), v);
        p[0] = v[0] * ld_x(x + c.x, pol);
        p[1] = v[1] * ld_x(x + c.y, pol);
        p[2] = v[2] * ld_x(x + c.z, pol);
        p[3] = v[3] * ld_x(x + c.w, pol);
    } else {
#pragma unroll
        for (int j = 0; j < kQ; ++j) {
            const int k = k0 + j;
            p[j] = k >= ea && k < eb ? ValueTraits<V>::f(ld_stream(vals + k)) * ld_x(x + ld_stream(colidx + k), pol)
                                     : 0.f;
        }
    }
}

// One tile: elements [tb, tb + kTile) of the run [ea, eb) (rows up to rb),
// lane l holding tb + 4l .. tb + 4l + 3 with products p. Each lane sums its
// elements row by row; a row wholly inside a lane is written by it; the
// parts of rows that cross lanes are joined by one segmented warp scan and
// written by the lane holding the row's last element; the row still open at
// the tile end is carried (open_row, carry). rcur is a row at or before the
// tile's first element.
__device__ __forceinline__ void csr_tile(int tb, int ea, int eb, int rb, const int* __restrict__ rowptr,
                                         float* __restrict__ y, const float (&p)[kQ], int lane, int& rcur,
                                         int& open_row, float& carry)
{
    const int k0 = tb + kQ * lane;
    const int klo = max(k0, ea), khi = min(k0 + kQ, eb) - 1;
    const bool any = klo <= khi;
    int nxt;
    int row = csr_row_of(rowptr, rcur, rb, eb, any ? klo : (k0 < ea ? ea : eb - 1), lane, &nxt);
    const int r0 = row;
    float s = 0.f, s_first = 0.f;
    bool multi = false;  // the first row ended inside the lane
#pragma unroll
    for (int j = 0; j < kQ; ++j) {
        const int k = k0 + j;
        if (k >= klo && k <= khi) {
            while (k >= nxt) {  // row `row` ended before k
                if (!multi) {
                    s_first = s;
                    multi = true;
                } else {
                    y[row] = s;  // began and ended inside this lane
                }
                s = 0.f;
                ++row;
                nxt = __ldg(rowptr + row + 1);
            }
            s += p[j];
        }
    }
    // row == the row of the lane's last element; nxt == its end
    const int r_last = any ? row : -1;
    const int prev = __shfl_up_sync(0xffffffffu, r_last, 1);
    const bool open_left = any && (lane == 0 ? open_row == r0 : prev == r0);
    const bool open_right = any && khi + 1 < nxt;
    // scan of the parts flowing right: a lane continues its left neighbour's
    // sum only when its single row came in from the left
    const bool reset = !(open_left && !multi);
    const float u = open_right ? s : 0.f;
    const unsigned rmask = __ballot_sync(0xffffffffu, reset);
    const int seg = 31 - __clz((rmask | 1u) & (0xffffffffu >> (31 - lane)));
    float f = u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(0xffffffffu, f, o);
        if (lane - o >= seg) f += t;
    }
    if (seg == 0 && !(rmask & 1u)) f += carry;
    float in = __shfl_up_sync(0xffffffffu, f, 1);
    if (lane == 0) in = carry;
    if (any) {
        if (multi) {
            y[r0] = open_left ? s_first + in : s_first;
            if (!open_right) y[row] = s;
        } else if (!open_right) {
            y[row] = open_left ? s + in : s;
        }
    }
    const bool o31 = __shfl_sync(0xffffffffu, open_right, 31);
    const float f31 = __shfl_sync(0xffffffffu, f, 31);
    const int r31 = __shfl_sync(0xffffffffu, r_last, 31);
    open_row = o31 ? r31 : -1;
    carry = o31 ? f31 : 0.f;
    if (r31 >= 0) rcur = r31;
}

// The rows [ra, rb) of one warp, none longer than kLongRow and at least one
// nonzero among them: tiles of kTile nonzeros from ea rounded down to a
// multiple of 4. Fixed tiles, fixed order: deterministic.
template <typename V, bool VEC>
__device__ __forceinline__ void csr_stream_rows(int ra, int rb, const int* __restrict__ rowptr,
                                                const int* __restrict__ colidx, const V* __restrict__ vals,
                                                const float* __restrict__ x, float* __restrict__ y, uint64_t pol,
                                                int lane)
{
    const int ea = __ldg(rowptr + ra), eb = __ldg(rowptr + rb);
    int rcur = ra, open_row = -1;
    float carry = 0.f;
    for (int base = ea & ~(kQ - 1); base < eb; base += kTile * kTiles) {
        float p[kTiles][kQ];
#pragma unroll
        for (int t = 0; t < kTiles; ++t) csr_quad<V, VEC>(colidx, vals, x, pol, base + t * kTile + kQ * lane, ea, eb, p[t]);
#pragma unroll
        for (int t = 0; t < kTiles; ++t) {
            const int tb = base + t * kTile;
            if (tb >= eb) break;
            csr_tile(tb, ea, eb, rb, rowptr, y, p[t], lane, rcur, open_row, carry);
        }
    }
}

// Smallest row i in [0, n] with i + rowptr[i] >= d: the row where the
// merge path of (rows, nonzeros) crosses diagonal d. Warp-wide 33-ary search.
__device__ __forceinline__ int csr_merge_row(const int* __restrict__ rowptr, int n, long long d, int lane)
{
    int lo = 0, hi = n;  // the answer lies in [lo, hi]; g(hi) >= d
    while (hi - lo > 32) {
        const long long span = hi - lo;
        const int q = lo + (int)(span * (lane + 1) / 33);  // strictly inside (lo, hi)
        const bool ge = (long long)q + __ldg(rowptr + q) >= d;
        const unsigned m = __ballot_sync(0xffffffffu, ge);
        const int f = m ? __ffs(m) - 1 : 32;  // first probe at or past d
        const int qf = __shfl_sync(0xffffffffu, q, f & 31);
        const int qp = __shfl_sync(0xffffffffu, q, (f + 31) & 31);
        if (f < 32) hi = qf;
        if (f > 0) lo = qp + 1;
    }
    const int q = lo + lane;
    const bool ge = q <= hi && (long long)q + __ldg(rowptr + q) >= d;
    const unsigned m = __ballot_sync(0xffffffffu, ge);
    return m ? lo + __ffs(m) - 1 : hi;
}

// Each warp owns the rows between two merge-path diagonals, an equal share
// of rows + nonzeros: empty rows are zeroed, rows longer than kLongRow go to
// the global list, the runs of other rows are streamed.
template <typename V, bool VEC>
__global__ void __launch_bounds__(256)
    csr_stream_kernel(int n, int nnz, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                      const V* __restrict__ vals, const float* __restrict__ x, float* __restrict__ y,
                      int* __restrict__ long_rows, int* __restrict__ n_long)
{
    const uint64_t pol = l2_evict_last_policy();
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long total = (long long)n + nnz;
    const int r0 = warp == 0 ? 0 : csr_merge_row(rowptr, n, total * warp / warps, lane);
    const int r1 = warp == warps - 1 ? n : csr_merge_row(rowptr, n, total * (warp + 1) / warps, lane);
    bool has_long = false;
    for (int r = r0 + lane; r < r1; r += 32) {
        const int len = __ldg(rowptr + r + 1) - __ldg(rowptr + r);
        if (len == 0) y[r] = 0.f;
        else if (len > kLongRow) {
            long_rows[atomicAdd(n_long, 1)] = r;
            has_long = true;
        }
    }
    if (!__any_sync(0xffffffffu, has_long)) {
        if (r1 > r0 && __ldg(rowptr + r1) > __ldg(rowptr + r0))
            csr_stream_rows<V, VEC>(r0, r1, rowptr, colidx, vals, x, y, pol, lane);
        return;
    }
    int r = r0;
    while (r < r1) {
        int rl = r1;  // next long row at or after r
        for (int rr = r; rr < r1; rr += 32) {
            const int q = rr + lane;
            const bool lg = q < r1 && __ldg(rowptr + q + 1) - __ldg(rowptr + q) > kLongRow;
            const unsigned m = __ballot_sync(0xffffffffu, lg);
            if (m) {
                rl = rr + __ffs(m) - 1;
                break;
            }
        }
        if (rl > r && __ldg(rowptr + rl) > __ldg(rowptr + r))
            csr_stream_rows<V, VEC>(r, rl, rowptr, colidx, vals, x, y, pol, lane);
        r = rl + 1;
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
#if CSR_STREAM
    {
        // equal merge-path shares, two per resident warp slot, at least 512
        // rows + nonzeros per warp
        static PerDeviceOnce occ_once;
        static std::atomic<int> occ{0};
        MR_CUDA_TRY(occ_once.run([&] {
            int b = 0;
            const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, csr_stream_kernel<V, true>, 256, 0);
            if (e == cudaSuccess) occ.store(std::max(1, b));
            return e;
        }));
        const long long total = (long long)n + nnz;
        const long long cap = (long long)sm_count() * std::max(1, occ.load()) * 2;
        const int grid = (int)std::max<long long>(1, std::min<long long>(cap, (total + 8 * 512 - 1) / (8 * 512)));
        const bool vec = (reinterpret_cast<uintptr_t>(colidx) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(vals) & (4 * sizeof(V) - 1)) == 0;
        if (vec)
            csr_stream_kernel<V, true><<<grid, 256, 0, st>>>(n, (int)nnz, rowptr, colidx, v, x, y, long_rows, n_long);
        else
            csr_stream_kernel<V, false><<<grid, 256, 0, st>>>(n, (int)nnz, rowptr, colidx, v, x, y, long_rows, n_long);
        MR_CUDA_TRY(cudaGetLastError());
        if (nnz > kLongRow) {
            const int lg = (int)std::max<int64_t>(1, std::min<int64_t>(max_long, (int64_t)sm_count() * 2));
            csr_long_rows_kernel<V><<<lg, kLongThreads, 0, st>>>(rowptr, colidx, v, x, y, long_rows, n_long);
            MR_CUDA_TRY(cudaGetLastError());
        }
        return MR_OK;
    }
#endif
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
