// Exact sector reuse-distance histogram on sm_100a.
//
// Reference (src/class.cu:864-936): walk the access stream s_k = colidx[k] /
// sector in order with a Fenwick tree over "last occurrence" positions; for
// each reuse k with previous occurrence p = prev[k], RD(k) = number of
// distinct sectors touched strictly between p and k; bin by upper_bound over
// the edges. That is inherently sequential (18 s median on R-MAT s24).
//
// Parallel restatement used here, exact in integers:
//   distinct sectors in (p, k) = #{b in (p, k) : prev[b] < p}
//   and, since every b <= p has prev[b] < b <= p,
//   RD(k) = L(k) - (p + 1)   with   L(k) = #{b < k : prev[b] < prev[k]}.
// L(k) is the per-element "smaller earlier values" count of the sequence
// prev[0..nnz), computed by a merge sort that carries a counter: whenever an
// element of the right (later) run is emitted, it adds the number of left-run
// elements already emitted. Non-negative prev values are distinct, so ties
// only occur among first touches (-1), which are never queried.
//
// Kernels: (1) sector keys; (2) stable LSD radix sort of (sector, position)
// in 8-bit digits -> prev[]; (3) 2048-element CTA merge sorts with counters
// in shared memory; (4) global merge passes (merge-path split per CTA,
// windows staged in shared memory); (5) binning with a shared-memory
// histogram and 64-bit atomics.
#include <algorithm>

#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096
constexpr int kRsBuckets = 256;

__global__ void sector_keys_kernel(const int32_t* __restrict__ s, int64_t n, int sector, uint32_t* __restrict__ key,
                                   int32_t* __restrict__ idx)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        key[k] = (uint32_t)(s[k] / sector);
        idx[k] = (int32_t)k;
    }
}

// per-tile digit histogram, digit-major layout hist[d * tiles + tile]
__global__ void __launch_bounds__(kRsThreads)
    radix_hist_kernel(const uint32_t* __restrict__ key, int64_t n, int shift, int tiles, int32_t* __restrict__ hist)
{
    __shared__ int cnt[kRsBuckets];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
    for (int i = threadIdx.x; i < kRsTile; i += kRsThreads)
        if (base + i < n) atomicAdd(&cnt[(key[base + i] >> shift) & 0xff], 1);
    __syncthreads();
    hist[(int64_t)threadIdx.x * tiles + blockIdx.x] = cnt[threadIdx.x];
}

// stable scatter: elements of a tile are ranked in order (round r, thread t)
// = position r*256 + t, using warp match + per-warp digit counts.
__global__ void __launch_bounds__(kRsThreads)
    radix_scatter_kernel(const uint32_t* __restrict__ key, const int32_t* __restrict__ val, int64_t n, int shift,
                         int tiles, const int32_t* __restrict__ offs, uint32_t* __restrict__ okey,
                         int32_t* __restrict__ oval)
{
    constexpr int W = kRsThreads / 32;
    __shared__ int running[kRsBuckets];
    __shared__ int wcnt[W][kRsBuckets];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    running[t] = offs[(int64_t)t * tiles + blockIdx.x];
    for (int j = 0; j < W; ++j) wcnt[j][t] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kRsItems; ++r) {
        const int64_t i = base + (int64_t)r * kRsThreads + t;
        const bool ok = i < n;
        const uint32_t k = ok ? key[i] : 0u;
        const int32_t v = ok ? val[i] : 0;
        const int d = ok ? (int)((k >> shift) & 0xff) : kRsBuckets + lane;  // unmatched sentinel
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (ok && rank == 0) wcnt[w][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            int pos = running[d] + rank;
            for (int j = 0; j < w; ++j) pos += wcnt[j][d];
            okey[pos] = k;
            oval[pos] = v;
        }
        __syncthreads();
        int add = 0;
        for (int j = 0; j < W; ++j) {
            add += wcnt[j][t];
            wcnt[j][t] = 0;
        }
        running[t] += add;
        __syncthreads();
    }
}

__global__ void prev_kernel(const uint32_t* __restrict__ key, const int32_t* __restrict__ idx, int64_t n,
                            int32_t* __restrict__ prev)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        prev[idx[i]] = (i > 0 && key[i - 1] == key[i]) ? idx[i - 1] : -1;
}

// ---------------------------------------------------------- merge count ----

constexpr int kMsThreads = 256;
constexpr int kMsItems = 8;
constexpr int kMsTile = kMsThreads * kMsItems;  // 2048

// number of A elements among the first d outputs of merge(A, B), ties to A
template <typename GetA, typename GetB>
__device__ __forceinline__ int merge_corank(GetA A, GetB B, int na, int nb, int d)
{
    int lo = max(0, d - nb), hi = min(d, na);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (A(mid) <= B(d - mid - 1))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// sorts each 2048-element tile of prev[] by value, carrying counters
__global__ void __launch_bounds__(kMsThreads)
    count_sort_tile_kernel(const int32_t* __restrict__ prev, int64_t n, int2* __restrict__ out)
{
    __shared__ int2 s[2][kMsTile];
    const int64_t base = (int64_t)blockIdx.x * kMsTile;
    const int tile_n = (int)min64(kMsTile, n - base);
    const int t = threadIdx.x;
    // thread-local: items [8t, 8t+8) in index order
    int v[kMsItems], c[kMsItems];
#pragma unroll
    for (int i = 0; i < kMsItems; ++i) {
        const int j = t * kMsItems + i;
        v[i] = (j < tile_n) ? prev[base + j] : INT32_MAX;  // padding sorts last
        c[i] = 0;
    }
#pragma unroll
    for (int i = 0; i < kMsItems; ++i)
#pragma unroll
        for (int j = 0; j < i; ++j) c[i] += (v[j] < v[i]) ? 1 : 0;
    // stable insertion sort of the 8 pairs by value
#pragma unroll
    for (int i = 1; i < kMsItems; ++i) {
#pragma unroll
        for (int j = i; j > 0; --j) {
            if (v[j - 1] > v[j]) {
                int tv = v[j], tc = c[j];
                v[j] = v[j - 1];
                c[j] = c[j - 1];
                v[j - 1] = tv;
                c[j - 1] = tc;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < kMsItems; ++i) s[0][t * kMsItems + i] = make_int2(v[i], c[i]);
    __syncthreads();
    int cur = 0;
    for (int run = kMsItems; run < kMsTile; run <<= 1) {
        const int2* src = s[cur];
        int2* dst = s[cur ^ 1];
        const int d0 = t * kMsItems;  // output position in the tile
        const int pair = d0 / (2 * run);
        const int lo = pair * 2 * run;
        const int2* A = src + lo;
        const int2* B = src + lo + run;
        const int d = d0 - lo;
        int a = merge_corank([&](int i) { return A[i].x; }, [&](int i) { return B[i].x; }, run, run, d);
        int b = d - a;
#pragma unroll
        for (int i = 0; i < kMsItems; ++i) {
            const bool takeA = (b >= run) || (a < run && A[a].x <= B[b].x);
            int2 e;
            if (takeA) {
                e = A[a++];
            } else {
                e = B[b++];
                e.y += a;
            }
            dst[d0 + i] = e;
        }
        __syncthreads();
        cur ^= 1;
    }
    // the whole tile is written (padding sorts to its end); out holds whole tiles
    for (int i = t; i < kMsTile; i += kMsThreads) out[base + i] = s[cur][i];
}

// one merge pass: runs of `run` elements (padded tail of INT32_MAX entries is
// never present: runs end at n). CTA b produces outputs [b*2048, b*2048+2048).
__global__ void __launch_bounds__(kMsThreads)
    count_merge_pass_kernel(const int2* __restrict__ in, int64_t n, int64_t run, int2* __restrict__ out)
{
    __shared__ int2 sA[kMsTile];
    __shared__ int2 sB[kMsTile];
    __shared__ int s_a0, s_a1;
    const int64_t d_begin = (int64_t)blockIdx.x * kMsTile;
    if (d_begin >= n) return;
    const int64_t pair_lo = (d_begin / (2 * run)) * 2 * run;
    const int64_t a_lo = pair_lo, a_hi = min64(pair_lo + run, n);
    const int64_t b_lo = a_hi, b_hi = min64(pair_lo + 2 * run, n);
    const int na = (int)(a_hi - a_lo), nb = (int)(b_hi - b_lo);
    const int dl = (int)(d_begin - pair_lo);
    const int dh = (int)min64(d_begin + kMsTile, b_hi) - (int)pair_lo;
    const int2* A = in + a_lo;
    const int2* B = in + b_lo;
    if (threadIdx.x == 0) s_a0 = merge_corank([&](int i) { return A[i].x; }, [&](int i) { return B[i].x; }, na, nb, dl);
    if (threadIdx.x == 32) s_a1 = merge_corank([&](int i) { return A[i].x; }, [&](int i) { return B[i].x; }, na, nb, dh);
    __syncthreads();
    const int a0 = s_a0, a1 = s_a1;
    const int b0 = dl - a0, b1 = dh - a1;
    const int wa = a1 - a0, wb = b1 - b0;
    for (int i = threadIdx.x; i < wa; i += kMsThreads) sA[i] = A[a0 + i];
    for (int i = threadIdx.x; i < wb; i += kMsThreads) sB[i] = B[b0 + i];
    __syncthreads();
    const int tot = wa + wb;
    const int d0 = min((int)threadIdx.x * kMsItems, tot);
    const int d1 = min(d0 + kMsItems, tot);
    int a = merge_corank([&](int i) { return sA[i].x; }, [&](int i) { return sB[i].x; }, wa, wb, d0);
    int b = d0 - a;
    for (int d = d0; d < d1; ++d) {
        const bool takeA = (b >= wb) || (a < wa && sA[a].x <= sB[b].x);
        int2 e;
        if (takeA) {
            e = sA[a++];
        } else {
            e = sB[b++];
            e.y += a0 + a;  // all of A's elements emitted before it in the whole pair
        }
        out[d_begin + d] = e;
    }
}

// RD = count - prev - 1 for reuses; histogram over the edges
__global__ void rd_bin_kernel(const int2* __restrict__ e, int64_t n, const int32_t* __restrict__ edges, int nedges,
                              unsigned long long* __restrict__ counts)
{
    __shared__ unsigned long long h[64];
    __shared__ int se[64];
    if (threadIdx.x < 64) {
        h[threadIdx.x] = 0;
        se[threadIdx.x] = threadIdx.x < nedges ? edges[threadIdx.x] : INT32_MAX;
    }
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int2 x = e[i];
        if (x.x < 0) continue;  // first touch: not a reuse
        const long long rd = (long long)x.y - x.x - 1;
        int b = 0;
        while (b < nedges && (long long)se[b] <= rd) ++b;
        atomicAdd(&h[b], 1ull);
    }
    __syncthreads();
    if (threadIdx.x <= nedges && h[threadIdx.x]) atomicAdd(&counts[threadIdx.x], h[threadIdx.x]);
}

int grid_of(int64_t n, int threads, int cap_per_sm = 16)
{
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, (int64_t)sm_count() * cap_per_sm));
}

}  // namespace

int radix_sort_pairs_u32(uint32_t*& keys, int32_t*& vals, uint32_t* kbuf, int32_t* vbuf, int64_t n, int bits,
                         cudaStream_t st)
{
    if (n <= 0) return MR_OK;
    const int tiles = (int)((n + kRsTile - 1) / kRsTile);
    DevBuf hist, scan_ws;
    MR_TRY(hist.alloc(sizeof(int32_t) * ((size_t)kRsBuckets * tiles + 1), st));
    MR_TRY(scan_ws.alloc(scan_workspace_bytes((int64_t)kRsBuckets * tiles), st));
    for (int shift = 0; shift < bits; shift += 8) {
        radix_hist_kernel<<<tiles, kRsThreads, 0, st>>>(keys, n, shift, tiles, hist.as<int32_t>());
        MR_TRY(exclusive_scan_i32_ws(hist.as<int32_t>(), hist.as<int32_t>(), (int64_t)kRsBuckets * tiles, scan_ws.p,
                                     st));
        radix_scatter_kernel<<<tiles, kRsThreads, 0, st>>>(keys, vals, n, shift, tiles, hist.as<int32_t>(), kbuf, vbuf);
        std::swap(keys, kbuf);
        std::swap(vals, vbuf);
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

int rd_hist_exact(const int32_t* stream, int64_t nnz, int32_t ncols, int32_t sector, const int32_t* edges,
                  int32_t nedges, int64_t* counts, int64_t* valid, cudaStream_t st)
{
    for (int b = 0; b <= nedges; ++b) counts[b] = 0;
    *valid = 0;
    if (nnz == 0) return MR_OK;
    const int64_t nsec = ((int64_t)ncols + sector - 1) / sector;
    int bits = 1;
    while (bits < 32 && ((int64_t)1 << bits) < nsec) ++bits;
    const int64_t ms_tiles = (nnz + kMsTile - 1) / kMsTile;

    DevBuf k0, k1, v0, v1, prev, m0, m1, dedges, dcounts;
    MR_TRY(k0.alloc(sizeof(uint32_t) * nnz, st));
    MR_TRY(k1.alloc(sizeof(uint32_t) * nnz, st));
    MR_TRY(v0.alloc(sizeof(int32_t) * nnz, st));
    MR_TRY(v1.alloc(sizeof(int32_t) * nnz, st));
    MR_TRY(dedges.alloc(sizeof(int32_t) * std::max(nedges, 1), st));
    MR_TRY(dcounts.alloc(sizeof(unsigned long long) * (nedges + 1), st));

    sector_keys_kernel<<<grid_of(nnz, 256), 256, 0, st>>>(stream, nnz, sector, k0.as<uint32_t>(), v0.as<int32_t>());
    uint32_t* ka = k0.as<uint32_t>();
    int32_t* va = v0.as<int32_t>();
    MR_TRY(radix_sort_pairs_u32(ka, va, k1.as<uint32_t>(), v1.as<int32_t>(), nnz, bits, st));
    MR_TRY(prev.alloc(sizeof(int32_t) * nnz, st));
    prev_kernel<<<grid_of(nnz, 256), 256, 0, st>>>(ka, va, nnz, prev.as<int32_t>());
    MR_TRY(m0.alloc(sizeof(int2) * (size_t)ms_tiles * kMsTile, st));
    MR_TRY(m1.alloc(sizeof(int2) * (size_t)ms_tiles * kMsTile, st));
    count_sort_tile_kernel<<<(int)ms_tiles, kMsThreads, 0, st>>>(prev.as<int32_t>(), nnz, m0.as<int2>());
    int2 *ma = m0.as<int2>(), *mb = m1.as<int2>();
    for (int64_t run = kMsTile; run < nnz; run *= 2) {
        count_merge_pass_kernel<<<(int)ms_tiles, kMsThreads, 0, st>>>(ma, nnz, run, mb);
        std::swap(ma, mb);
    }
    MR_CUDA_TRY(cudaGetLastError());
    MR_CUDA_TRY(cudaMemcpyAsync(dedges.p, edges, sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st));
    MR_CUDA_TRY(cudaMemsetAsync(dcounts.p, 0, sizeof(unsigned long long) * (nedges + 1), st));
    rd_bin_kernel<<<grid_of(nnz, 256, 8), 256, 0, st>>>(ma, nnz, dedges.as<int32_t>(), nedges,
                                                      dcounts.as<unsigned long long>());
    MR_CUDA_TRY(cudaGetLastError());
    MR_CUDA_TRY(cudaMemcpyAsync(counts, dcounts.p, sizeof(int64_t) * (nedges + 1), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    int64_t tot = 0;
    for (int b = 0; b <= nedges; ++b) tot += counts[b];
    *valid = tot;
    return MR_OK;
}

}  // namespace mr
