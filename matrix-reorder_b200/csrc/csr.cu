// Plain CSR SpMV for sm_100a (the reference's cuSPARSE CSR_ALG1 path,
// src/class.cu:1359-1397, replaced by a hand-written kernel).
//
// Two kernels, both deterministic (every sum is formed in a fixed order that
// does not depend on timing):
//  * csr_stream_kernel: every warp owns the rows between two merge-path
//    diagonals of (rows, nonzeros), an equal share of both, found by a
//    warp-wide 33-ary search of i + rowptr[i]. Its nonzeros are streamed in
//    tiles of 128, four consecutive nonzeros per lane (16-byte evict-first
//    loads of colidx and values, x gathered through L2 with an evict-last
//    policy); the next tile's loads are issued before the current tile is
//    summed. Each lane finds the row of its first nonzero by a shuffle
//    search over the next 32 row starts, sums its nonzeros row by row and
//    writes the rows that lie inside it; the parts of rows that cross lanes
//    are joined by one segmented warp scan and written by the lane holding
//    the row's last nonzero, and the row open at the tile end is carried to
//    the next tile. Empty rows are zeroed; rows longer than kLongRow are
//    skipped and appended to a global list.
//  * csr_long_rows_kernel: one 1024-thread CTA per listed row, a fixed
//    per-thread stride (four loads in flight) and a fixed shared-memory tree.
#include <atomic>
#include <climits>

#include "common.cuh"
#include "internal.hpp"

namespace mr {

constexpr int kLongRow = 4096;
constexpr int kLongThreads = 1024;
constexpr int kQ = 4;               // consecutive nonzeros per lane in a tile
constexpr int kTileNnz = 32 * kQ;   // nonzeros per warp tile
constexpr int kWarpsPerCta = 4;  // small CTAs: more of them resident, finer tail

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

// Products of the Q nonzeros k0 .. k0+Q-1 (zero outside [ea, eb)); whole
// groups of four in range are vector loads.
// Column indices and values of the Q nonzeros k0 .. k0+Q-1; outside
// [ea, eb) the column is -1.
template <typename V, bool VEC, int Q>
__device__ __forceinline__ void csr_ld_stream(const int* __restrict__ colidx, const V* __restrict__ vals, int k0,
                                              int ea, int eb, int (&c)[Q], float (&w)[Q])
{
    if (VEC && k0 >= ea && k0 + Q <= eb) {
#pragma unroll
        for (int i = 0; i < Q / 4; ++i) {
            const int4 ci = ld_stream(reinterpret_cast<const int4*>(colidx + k0) + i);
            float v[4];
            Vec4<V>::unpack(ld_stream(reinterpret_cast<const typename Vec4<V>::T*>(vals + k0) + i), v);
            c[4 * i + 0] = ci.x;
            c[4 * i + 1] = ci.y;
            c[4 * i + 2] = ci.z;
            c[4 * i + 3] = ci.w;
#pragma unroll
            for (int j = 0; j < 4; ++j) w[4 * i + j] = v[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            const int k = k0 + j;
            const bool in = k >= ea && k < eb;
            c[j] = in ? ld_stream(colidx + k) : -1;
            w[j] = in ? ValueTraits<V>::f(ld_stream(vals + k)) : 0.f;
        }
    }
}

// One tile: elements [tb, tb + 32Q) of the run [ea, eb) (rows up to rb),
// lane l holding tb + Ql .. tb + Ql + Q-1 with products p. Each lane sums its
// elements row by row; a row wholly inside a lane is written by it; the
// parts of rows that cross lanes are joined by one segmented warp scan and
// written by the lane holding the row's last element; the row still open at
// the tile end is carried (open_row, carry). rcur is a row at or before the
// tile's first element.
template <int Q>
__device__ __forceinline__ void csr_tile(int tb, int ea, int eb, int rb, const int* __restrict__ rowptr,
                                         float* __restrict__ y, const float (&p)[Q], int lane, int& rcur,
                                         int& open_row, float& carry)
{
    const int k0 = tb + Q * lane;
    const int klo = max(k0, ea), khi = min(k0 + Q, eb) - 1;
    const bool any = klo <= khi;
    int nxt;
    int row = csr_row_of(rowptr, rcur, rb, eb, any ? klo : (k0 < ea ? ea : eb - 1), lane, &nxt);
    const int r0 = row;
    float s = 0.f, s_first = 0.f;
    bool multi = false;  // the first row ended inside the lane
#pragma unroll
    for (int j = 0; j < Q; ++j) {
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

// The rows [ra, rb) of one warp, none longer than kLongRow, at least one
// nonzero among them: tiles of kTileNnz nonzeros from ea rounded down to a
// multiple of 4, the next tile's index and value loads in flight while the
// current tile is summed. Fixed tiles, fixed order: deterministic.
template <typename V, bool VEC>
__device__ __forceinline__ void csr_stream_rows(int ra, int rb, const int* __restrict__ rowptr,
                                                const int* __restrict__ colidx, const V* __restrict__ vals,
                                                const float* __restrict__ x, float* __restrict__ y, uint64_t pol,
                                                int lane)
{
    const int ea = __ldg(rowptr + ra), eb = __ldg(rowptr + rb);
    int rcur = ra, open_row = -1;
    float carry = 0.f;
    int c[kQ];
    float w[kQ];
    csr_ld_stream<V, VEC, kQ>(colidx, vals, (ea & ~3) + kQ * lane, ea, eb, c, w);
    for (int base = ea & ~3; base < eb; base += kTileNnz) {
        float p[kQ];
#pragma unroll
        for (int j = 0; j < kQ; ++j) p[j] = c[j] >= 0 ? w[j] * ld_x(x + c[j], pol) : 0.f;
        if (base + kTileNnz < eb) csr_ld_stream<V, VEC, kQ>(colidx, vals, base + kTileNnz + kQ * lane, ea, eb, c, w);
        csr_tile<kQ>(base, ea, eb, rb, rowptr, y, p, lane, rcur, open_row, carry);
    }
}

// For each of two diagonals d: the smallest row i in [0, n] with
// i + rowptr[i] >= d, the row where the merge path of (rows, nonzeros)
// crosses d. Warp-wide 33-ary searches (the answer lies in [lo, hi], with
// g(hi) >= d), the two in lockstep: their probes are issued together, so the
// warp waits for one chain of dependent loads instead of two.
__device__ __forceinline__ int2 csr_merge_rows2(const int* __restrict__ rowptr, int n, long long d0, long long d1,
                                                int lane)
{
    int lo[2] = {0, 0}, hi[2] = {n, n};
    const long long d[2] = {d0, d1};
    while (hi[0] - lo[0] > 32 || hi[1] - lo[1] > 32) {
        int q[2];
        bool ge[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const long long span = hi[k] - lo[k];
            q[k] = lo[k] + (int)(span * (lane + 1) / 33);
            ge[k] = span > 32 && (long long)q[k] + __ldg(rowptr + q[k]) >= d[k];
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (hi[k] - lo[k] <= 32) continue;  // this search is done (warp-uniform)
            const unsigned m = __ballot_sync(0xffffffffu, ge[k]);
            const int f = m ? __ffs(m) - 1 : 32;
            const int qf = __shfl_sync(0xffffffffu, q[k], f & 31);
            const int qp = __shfl_sync(0xffffffffu, q[k], (f + 31) & 31);
            if (f < 32) hi[k] = qf;
            if (f > 0) lo[k] = qp + 1;
        }
    }
    int r[2];
    bool ge[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int q = lo[k] + lane;
        ge[k] = q <= hi[k] && (long long)q + __ldg(rowptr + q) >= d[k];
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const unsigned m = __ballot_sync(0xffffffffu, ge[k]);
        r[k] = m ? lo[k] + __ffs(m) - 1 : hi[k];
    }
    return make_int2(r[0], r[1]);
}

// Each warp owns the rows between two merge-path diagonals, an equal share
// of rows + nonzeros: empty rows are zeroed, rows longer than kLongRow go to
// the global list, the runs of other rows are streamed.
template <typename V, bool VEC>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
    csr_stream_kernel(int n, int nnz, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                      const V* __restrict__ vals, const float* __restrict__ x, float* __restrict__ y,
                      int* __restrict__ long_rows, int* __restrict__ n_long)
{
    const uint64_t pol = l2_evict_last_policy();
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long total = (long long)n + nnz;
    const int2 rr = csr_merge_rows2(rowptr, n, total * warp / warps, total * (warp + 1) / warps, lane);
    const int r0 = warp == 0 ? 0 : rr.x;
    const int r1 = warp == warps - 1 ? n : rr.y;
    // row lengths 128 rows at a time, every load of a round in flight
    bool has_long = false;
    for (int base = r0; base < r1; base += 4 * 32) {
        int len[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = base + lane + 32 * j;
            len[j] = r < r1 ? __ldg(rowptr + r + 1) - __ldg(rowptr + r) : 1;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = base + lane + 32 * j;
            if (r >= r1) continue;
            if (len[j] == 0) y[r] = 0.f;
            else if (len[j] > kLongRow) {
                long_rows[atomicAdd(n_long, 1)] = r;
                has_long = true;
            }
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
    const long long total = (long long)n + nnz;
    // four merge-path shares per resident warp (shorter shares even out the
    // tail: +2% over two at R-MAT s22), at least 512 rows + nonzeros each
    static PerDeviceOnce occ_once;
    static std::atomic<int> occ{0};
    MR_CUDA_TRY(occ_once.run([&] {
        int b = 0;
        const cudaError_t e =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, csr_stream_kernel<V, true>, kWarpsPerCta * 32, 0);
        if (e == cudaSuccess) occ.store(std::max(1, b));
        return e;
    }));
    const long long cap = (long long)sm_count() * std::max(1, occ.load()) * 4;
    const long long per_cta = (long long)kWarpsPerCta * 512;
    const int grid = (int)std::max<long long>(1, std::min<long long>(cap, (total + per_cta - 1) / per_cta));
    const bool vec = (reinterpret_cast<uintptr_t>(colidx) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(vals) & (4 * sizeof(V) - 1)) == 0;
    if (vec)
        csr_stream_kernel<V, true><<<grid, kWarpsPerCta * 32, 0, st>>>(n, (int)nnz, rowptr, colidx, v, x, y,
                                                                      long_rows, n_long);
    else
        csr_stream_kernel<V, false><<<grid, kWarpsPerCta * 32, 0, st>>>(n, (int)nnz, rowptr, colidx, v, x, y,
                                                                       long_rows, n_long);
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
