// Applying a permutation to a CSR matrix on sm_100a: B = P A P^T.
//
// Reference semantics (src/class.cu:2686-2705): perm[old] = new is scattered
// from the ordering, both COO index arrays are gathered through perm, and
// GRAPH::sort(false) (src/class.cu:423-457) re-sorts all nnz by (new row, new
// column) with a comparator merge sort; coo2csr (src/class.cu:1342) rebuilds
// the row pointer.
//
// Here the row structure is kept: new row i is old row inv[i], so the new
// row pointer is an exclusive scan of the gathered row lengths, and only the
// columns inside each row need sorting. Each row is sorted by the 64-bit key
// (new column << 32 | position in the source row), which makes the order
// unique and keeps equal columns in source order; the value is fetched
// through the position after the sort. Rows go to one of three sorters by
// length: a 32-lane shuffle bitonic network (<= 32), a shared-memory bitonic
// sort in one CTA (<= 4096), or a CTA-wide chunked merge sort through global
// scratch (longer rows).
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace mr {

// ------------------------------------------------------------ scan --------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int& total)
{
    const int lid = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lid >= o) x += t;
    }
    if (lid == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = (lid < kScanThreads / 32) ? s_warp[lid] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lid >= o) w += t;
        }
        if (lid < kScanThreads / 32) s_warp[lid] = w;  // inclusive warp totals
    }
    __syncthreads();
    total = s_warp[kScanThreads / 32 - 1];
    const int before = wid ? s_warp[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const int32_t* __restrict__ in, int64_t n,
                                                                    int32_t* __restrict__ partial)
{
    __shared__ int s_warp[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int s = 0;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads)
        if (base + i < n) s += in[base + i];
    int total;
    block_exclusive_scan(s, s_warp, total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// single CTA: exclusive scan of the per-tile sums, chunk by chunk
__global__ void __launch_bounds__(kScanThreads) scan_partials_kernel(int32_t* __restrict__ partial, int nb)
{
    __shared__ int s_warp[kScanThreads / 32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        const int i = b0 + threadIdx.x;
        const int v = (i < nb) ? partial[i] : 0;
        int total;
        const int ex = block_exclusive_scan(v, s_warp, total);
        if (i < nb) partial[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const int32_t* in, int64_t n,
                                                                   const int32_t* __restrict__ partial, int32_t* out)
{
    __shared__ int s_tile[kScanTile];
    __shared__ int s_warp[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) s_tile[i] = (base + i < n) ? in[base + i] : 0;
    __syncthreads();
    int local[kScanItems];
    int s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        local[j] = s_tile[threadIdx.x * kScanItems + j];
        s += local[j];
    }
    int total;
    int ex = block_exclusive_scan(s, s_warp, total) + partial[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        s_tile[threadIdx.x * kScanItems + j] = ex;
        ex += local[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads)
        if (base + i < n) out[base + i] = s_tile[i];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = partial[blockIdx.x] + total;
}

size_t scan_workspace_bytes(int64_t n) { return sizeof(int32_t) * (size_t)((n + kScanTile - 1) / kScanTile + 1); }

int exclusive_scan_i32_ws(const int32_t* in, int32_t* out, int64_t n, void* ws, cudaStream_t st)
{
    if (n <= 0) {
        MR_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int32_t), st));
        return MR_OK;
    }
    const int nb = (int)((n + kScanTile - 1) / kScanTile);
    int32_t* partial = reinterpret_cast<int32_t*>(ws);
    scan_reduce_kernel<<<nb, kScanThreads, 0, st>>>(in, n, partial);
    scan_partials_kernel<<<1, kScanThreads, 0, st>>>(partial, nb);
    scan_apply_kernel<<<nb, kScanThreads, 0, st>>>(in, n, partial, out);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

int exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t st)
{
    DevBuf ws;
    MR_TRY(ws.alloc(scan_workspace_bytes(n), st));
    return exclusive_scan_i32_ws(in, out, n, ws.p, st);
}

// ------------------------------------------------------ permutations ------

__global__ void perm_invert_kernel(int n, const int32_t* __restrict__ perm, int32_t* __restrict__ inv, int* bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = perm[i];
        if (p < 0 || p >= n)
            atomicOr(bad, 1);
        else
            inv[p] = i;
    }
}

// After inv was filled with -1 and scattered: any hole means perm is not a
// bijection (a repeated value leaves some slot unwritten).
__global__ void perm_holes_kernel(int n, const int32_t* __restrict__ inv, int* bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (inv[i] < 0) atomicOr(bad, 1);
}

static int grid_for(int64_t n, int threads) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, (int64_t)sm_count() * 16)); }

int launch_perm_invert(int n, const int32_t* perm, int32_t* inv, int* bad_flag, cudaStream_t st)
{
    MR_CUDA_TRY(cudaMemsetAsync(inv, 0xff, sizeof(int32_t) * (size_t)n, st));
    perm_invert_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, perm, inv, bad_flag);
    perm_holes_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, inv, bad_flag);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

int check_perm(const int32_t* perm, int n, int* valid, cudaStream_t st)
{
    DevBuf inv, flag;
    MR_TRY(inv.alloc(sizeof(int32_t) * (size_t)std::max(n, 1), st));
    MR_TRY(flag.alloc(sizeof(int), st));
    MR_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    if (n > 0) MR_TRY(launch_perm_invert(n, perm, inv.as<int32_t>(), flag.as<int>(), st));
    int h = 0;
    MR_CUDA_TRY(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    *valid = (h == 0);
    return MR_OK;
}

// A block covers kPvPer * 256 consecutive elements, thread t the elements
// t, t + 256, ...: the thread loads its kPvPer permutation entries, then its
// kPvPer inputs, then stores, so that kPvPer independent loads are in flight
// per thread at each step (the random side, the gather of the inverse or the
// scatter of the forward permutation, is the latency-bound one).
constexpr int kPvPer = 4;

__global__ void __launch_bounds__(256) permute_vector_kernel(int n, const int32_t* __restrict__ perm,
                                                             const float* __restrict__ in, float* __restrict__ out,
                                                             int inverse)
{
    const int64_t base = (int64_t)blockIdx.x * (256 * kPvPer) + threadIdx.x;
    int p[kPvPer];
    float v[kPvPer];
#pragma unroll
    for (int e = 0; e < kPvPer; ++e) {
        const int64_t i = base + 256 * e;
        p[e] = i < n ? __ldg(perm + i) : -1;
        if (p[e] >= n) p[e] = -1;  // not a permutation entry: skipped
    }
#pragma unroll
    for (int e = 0; e < kPvPer; ++e) {
        const int64_t i = base + 256 * e;
        v[e] = p[e] < 0 ? 0.f : (inverse ? __ldg(in + p[e]) : __ldg(in + i));
    }
#pragma unroll
    for (int e = 0; e < kPvPer; ++e) {
        const int64_t i = base + 256 * e;
        if (p[e] < 0) continue;
        if (inverse)
            out[i] = v[e];
        else
            out[p[e]] = v[e];
    }
}

int launch_permute_vector(int n, const int32_t* perm, const float* in, float* out, int inverse, cudaStream_t st)
{
    if (n <= 0) return MR_OK;
    const int grid = (int)(((int64_t)n + 256 * kPvPer - 1) / (256 * kPvPer));
    permute_vector_kernel<<<grid, 256, 0, st>>>(n, perm, in, out, inverse);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

// ------------------------------------------------------------ validate ----

// bad |= 1: rowptr[0] != 0, rowptr decreasing or rowptr[n] != nnz;
// bad |= 2: a column index outside [0, ncols).
__global__ void validate_rowptr_kernel(int n, int64_t nnz, const int32_t* __restrict__ rowptr, int* bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        const int v = rowptr[i];
        if ((i == 0 && v != 0) || (i == n && (int64_t)v != nnz) || (i < n && rowptr[i + 1] < v)) atomicOr(bad, 1);
    }
}

__global__ void validate_colidx_kernel(int64_t nnz, int ncols, const int32_t* __restrict__ colidx, int* bad)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int c = colidx[k];
        if (c < 0 || c >= ncols) atomicOr(bad, 2);
    }
}

int validate_csr_async(const mr_csr_view& A, int* bad_dev, cudaStream_t st)
{
    validate_rowptr_kernel<<<grid_for((int64_t)A.n_rows + 1, 256), 256, 0, st>>>(A.n_rows, A.nnz, A.rowptr, bad_dev);
    if (A.nnz > 0)
        validate_colidx_kernel<<<grid_for(A.nnz, 256), 256, 0, st>>>(A.nnz, A.n_cols, A.colidx, bad_dev);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

int validate_csr(const mr_csr_view& A, int* ok, cudaStream_t st)
{
    DevBuf flag;
    MR_TRY(flag.alloc(sizeof(int), st));
    MR_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    MR_TRY(validate_csr_async(A, flag.as<int>(), st));
    int h = 0;
    MR_CUDA_TRY(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    *ok = (h == 0);
    return MR_OK;
}

// --------------------------------------------------------- CSR permute ----

constexpr int kTinyRow = 8;     // one thread, a sorting network in registers
constexpr int kSmallRow = 32;   // one warp, one key per lane
constexpr int kWarpRow = 256;   // one warp, up to 8 keys per lane in registers
constexpr int kMedRow = 4096;   // one CTA, shared-memory bitonic; longer rows: chunks + merge passes

struct PermStats {
    int bad;
    int bad_csr;
    int max_len;
    int n_small;
    int n_warp;
    int n_med;
    int n_large;
    unsigned long long large_total;
};

// new row lengths and the lists of rows that need more than one key per
// lane (warp-aggregated appends: one atomic per warp and list)
__global__ void __launch_bounds__(256)
    row_lengths_kernel(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ inv,
                       int32_t* __restrict__ len, PermStats* stats, int32_t* __restrict__ small_list,
                       int32_t* __restrict__ warp_list, int32_t* __restrict__ med_list,
                       int32_t* __restrict__ large_list)
{
    // list appends: ranks within the warp (ballot), warp offsets within the
    // CTA (shared counters), one global atomic per class and CTA step. The
    // order of a list only decides which CTA sorts which row.
    __shared__ int s_cnt[4], s_base[4];
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int i = base + (int)threadIdx.x;
        int l = 0;
        if (i < n) {
            const int o = inv[i];
            if (o >= 0 && o < n) l = rowptr[o + 1] - rowptr[o];
            len[i] = l;
        }
        // 0: empty or at most kTinyRow keys (no list: the tiny kernel visits every row)
        const int cls = (i >= n || l <= kTinyRow)
                            ? 0
                            : (l <= kSmallRow ? 4 : (l <= kWarpRow ? 1 : (l <= kMedRow ? 2 : 3)));
        if (cls == 3) {
            atomicMax(&stats->max_len, l);
            atomicAdd(&stats->large_total, (unsigned long long)l);
        }
        if (threadIdx.x < 4) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        int warp_off[4], rank = 0;
#pragma unroll
        for (int c = 1; c <= 4; ++c) {
            const unsigned m = __ballot_sync(0xffffffffu, cls == c);
            int off = 0;
            if (m && lane == __ffs(m) - 1) off = atomicAdd(&s_cnt[c - 1], __popc(m));
            warp_off[c - 1] = __shfl_sync(0xffffffffu, off, m ? __ffs(m) - 1 : 0);
            if (cls == c) rank = __popc(m & ((1u << lane) - 1u));
        }
        __syncthreads();
        if (threadIdx.x < 4 && s_cnt[threadIdx.x] > 0) {
            const int c = threadIdx.x + 1;
            int* counter = c == 1 ? &stats->n_warp : (c == 2 ? &stats->n_med : (c == 3 ? &stats->n_large : &stats->n_small));
            s_base[threadIdx.x] = atomicAdd(counter, s_cnt[threadIdx.x]);
        }
        __syncthreads();
        if (cls > 0) {
            int32_t* list = cls == 1 ? warp_list : (cls == 2 ? med_list : (cls == 3 ? large_list : small_list));
            list[s_base[cls - 1] + warp_off[cls - 1] + rank] = i;
        }
        __syncthreads();  // s_cnt / s_base are reset by the next step
    }
}

// key = (new column << 32) | position in the source row: unique, so every
// sort below is deterministic and keeps equal columns in source order
__device__ __forceinline__ unsigned long long perm_key(const int32_t* __restrict__ perm, const int32_t* __restrict__ colidx,
                                                       int src, int t)
{
    return ((unsigned long long)(uint32_t)__ldg(perm + __ldg(colidx + src + t)) << 32) | (unsigned)t;
}

template <typename E>
__device__ __forceinline__ void emit_sorted(unsigned long long key, int dst, int src, const E* __restrict__ vals,
                                            int32_t* __restrict__ out_col, E* __restrict__ out_val)
{
    out_col[dst] = (int32_t)(key >> 32);
    out_val[dst] = vals[src + (int)(key & 0xffffffffu)];
}

// rows of length <= 32: one warp per row, bitonic network in registers
// compare-exchange: a <= b afterwards
__device__ __forceinline__ void cx(unsigned long long& a, unsigned long long& b)
{
    const unsigned long long lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

// rows of 1 .. kTinyRow keys: one thread per row, keys padded with ~0 to a
// sorting network of 4 (5 exchanges) or 8 (19 exchanges, Batcher's
// odd-even merge sort) in registers
template <typename E>
__global__ void __launch_bounds__(256)
    sort_tiny_rows_kernel(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                          const E* __restrict__ vals, const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                          const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                          E* __restrict__ out_val)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        if (len == 0 || len > kTinyRow) continue;
        const int src = rowptr[inv[i]];
        unsigned long long k[kTinyRow];
#pragma unroll
        for (int j = 0; j < kTinyRow; ++j) k[j] = j < len ? perm_key(perm, colidx, src, j) : ~0ull;
        if (len > 1) {
            cx(k[0], k[1]);
            cx(k[2], k[3]);
            cx(k[0], k[2]);
            cx(k[1], k[3]);
            cx(k[1], k[2]);
            if (len > 4) {
                cx(k[4], k[5]);
                cx(k[6], k[7]);
                cx(k[4], k[6]);
                cx(k[5], k[7]);
                cx(k[5], k[6]);
                // merge the two sorted halves
                cx(k[0], k[4]);
                cx(k[1], k[5]);
                cx(k[2], k[6]);
                cx(k[3], k[7]);
                cx(k[2], k[4]);
                cx(k[3], k[5]);
                cx(k[1], k[2]);
                cx(k[3], k[4]);
                cx(k[5], k[6]);
            }
        }
#pragma unroll
        for (int j = 0; j < kTinyRow; ++j)
            if (j < len) emit_sorted<E>(k[j], dst + j, src, vals, out_col, out_val);
    }
}

// rows of kTinyRow+1 .. kSmallRow keys (listed): one warp each, one key per
// lane, a register bitonic network over the warp
template <typename E>
__global__ void __launch_bounds__(256)
    sort_small_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                           const int32_t* __restrict__ colidx, const E* __restrict__ vals,
                           const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                           const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                           E* __restrict__ out_val)
{
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < count; r += warps) {
        const int i = list[r];
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        const int src = rowptr[inv[i]];
        unsigned long long key = ~0ull;
        if (lane < len) key = perm_key(perm, colidx, src, lane);
#pragma unroll
        for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, j);
                const bool up = (lane & k) == 0;
                const bool lower = (lane & j) == 0;
                key = (lower == up) ? min(key, other) : max(key, other);
            }
        }
        if (lane < len) emit_sorted<E>(key, dst + lane, src, vals, out_col, out_val);
    }
}

// Bitonic stages j = jtop, jtop/2, ..., 1 of merge size `size` on 32*R
// keys held by one warp in striped order: key r of lane l is element
// base + r*32 + l of the network (base: the warp's first element), so the
// compare directions are those of the whole network. Distances below 32
// exchange across lanes, larger ones inside a thread's registers.
template <int R>
__device__ __forceinline__ void warp_stages(unsigned long long (&k)[R], int lane, int base, int size, int jtop)
{
    constexpr int LOG = R >= 16 ? 8 : (R >= 8 ? 7 : (R >= 4 ? 6 : (R >= 2 ? 5 : 4)));  // log2(32 R) - 1
#pragma unroll
    for (int jj = LOG; jj >= 0; --jj) {
        const int j = 1 << jj;
        if (j > jtop) continue;
        if (j >= 32) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int p = r ^ (j >> 5);
                if (p > r) {
                    const bool up = ((base + r * 32 + lane) & size) == 0;
                    const unsigned long long a = k[r], b = k[p];
                    const bool sw = up ? (a > b) : (a < b);
                    k[r] = sw ? b : a;
                    k[p] = sw ? a : b;
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const bool up = ((base + r * 32 + lane) & size) == 0;
                const bool lower = (lane & j) == 0;
                const unsigned long long o = __shfl_xor_sync(0xffffffffu, k[r], j);
                k[r] = (lower == up) ? min(k[r], o) : max(k[r], o);
            }
        }
    }
}

// full bitonic sort of the warp's 32*R keys (as part of a network whose
// element base is the warp's first)
template <int R> __device__ __forceinline__ void warp_bitonic(unsigned long long (&k)[R], int lane, int base)
{
#pragma unroll
    for (int size = 2; size <= 32 * R; size <<= 1) warp_stages<R>(k, lane, base, size, size >> 1);
}

// Bitonic sort of 256*R keys by a 256-thread CTA: every warp sorts its 32*R
// keys in registers, then each merge size above a warp's span runs its long
// distances through shared memory (s[256*R]) and the rest in registers.
template <int R>
__device__ __forceinline__ void cta_bitonic_regs(unsigned long long (&k)[R], unsigned long long* s, int warp, int lane)
{
    constexpr int WS = 32 * R;
    constexpr int P = 8 * WS;
    const int base = warp * WS;
    warp_bitonic<R>(k, lane, base);
#pragma unroll
    for (int size = 2 * WS; size <= P; size <<= 1) {
#pragma unroll
        for (int r = 0; r < R; ++r) s[base + r * 32 + lane] = k[r];
        __syncthreads();
        for (int j = size >> 1; j >= WS; j >>= 1) {
            for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const int i = (t / j) * 2 * j + (t % j);  // bit j of i clear
                const int q = i + j;
                const bool up = (i & size) == 0;
                const unsigned long long a = s[i], b = s[q];
                if ((a > b) == up) {
                    s[i] = b;
                    s[q] = a;
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < R; ++r) k[r] = s[base + r * 32 + lane];
        __syncthreads();  // s is rewritten by the next merge size
        warp_stages<R>(k, lane, base, size, WS >> 1);
    }
}

template <typename E, int R>
__device__ __forceinline__ void warp_row_sort(int len, int src, int dst, const int32_t* __restrict__ colidx,
                                              const E* __restrict__ vals, const int32_t* __restrict__ perm,
                                              int32_t* __restrict__ out_col, E* __restrict__ out_val, int lane)
{
    unsigned long long k[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = r * 32 + lane;
        k[r] = t < len ? perm_key(perm, colidx, src, t) : ~0ull;
    }
    warp_bitonic<R>(k, lane, 0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = r * 32 + lane;
        if (t < len) emit_sorted<E>(k[r], dst + t, src, vals, out_col, out_val);
    }
}

// rows of length (32, 256]: one warp per row, 2 to 8 keys per lane (a
// 16-key network unrolled in the same kernel costs more in instruction
// fetch than it saves)
template <typename E>
__global__ void __launch_bounds__(256, 3)
    sort_warp_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                          const int32_t* __restrict__ colidx, const E* __restrict__ vals,
                          const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                          const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                          E* __restrict__ out_val)
{
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
        const int i = list[w];
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        const int src = rowptr[inv[i]];
        if (len <= 64)
            warp_row_sort<E, 2>(len, src, dst, colidx, vals, perm, out_col, out_val, lane);
        else if (len <= 128)
            warp_row_sort<E, 4>(len, src, dst, colidx, vals, perm, out_col, out_val, lane);
        else
            warp_row_sort<E, 8>(len, src, dst, colidx, vals, perm, out_col, out_val, lane);
    }
}

// keys [0, cnt) of a row segment (positions start + t), sorted by one CTA
// with 256*R slots, handed to `sink(t, key)` in order
template <int R, typename F>
__device__ __forceinline__ void cta_sort_segment(int cnt, int src, int start, const int32_t* __restrict__ colidx,
                                                 const int32_t* __restrict__ perm, unsigned long long* s, F&& sink)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long k[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = warp * 32 * R + r * 32 + lane;
        k[r] = t < cnt ? perm_key(perm, colidx, src, start + t) : ~0ull;
    }
    cta_bitonic_regs<R>(k, s, warp, lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = warp * 32 * R + r * 32 + lane;
        if (t < cnt) sink(t, k[r]);
    }
}

template <typename F>
__device__ __forceinline__ void cta_sort_any(int cnt, int src, int start, const int32_t* __restrict__ colidx,
                                             const int32_t* __restrict__ perm, unsigned long long* s, F&& sink)
{
    if (cnt <= 512)
        cta_sort_segment<2>(cnt, src, start, colidx, perm, s, sink);
    else if (cnt <= 1024)
        cta_sort_segment<4>(cnt, src, start, colidx, perm, s, sink);
    else if (cnt <= 2048)
        cta_sort_segment<8>(cnt, src, start, colidx, perm, s, sink);
    else
        cta_sort_segment<16>(cnt, src, start, colidx, perm, s, sink);
}

// rows of length (256, 4096]: one 256-thread CTA per row (grid-stride over
// the list). Two instantiations: rows of at most kMedSmall keys with a small
// buffer and 6 CTAs per SM, the longer ones with the full buffer at 2 per SM
// (each skips the other's rows).
constexpr int kMedSmall = 1024;

template <typename E, int MAXLEN>
__global__ void __launch_bounds__(256, MAXLEN <= kMedSmall ? 6 : 2)
    sort_med_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                         const int32_t* __restrict__ colidx, const E* __restrict__ vals,
                         const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                         const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                         E* __restrict__ out_val)
{
    __shared__ unsigned long long s[MAXLEN];
    for (int r = blockIdx.x; r < count; r += gridDim.x) {
        const int i = list[r];
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        if ((len <= kMedSmall) != (MAXLEN <= kMedSmall)) continue;  // the other instantiation's row
        const int src = rowptr[inv[i]];
        // sorted keys back to shared memory, then a coalesced emit
        if constexpr (MAXLEN <= kMedSmall) {
            if (len <= 512)
                cta_sort_segment<2>(len, src, 0, colidx, perm, s, [&](int t, unsigned long long key) { s[t] = key; });
            else
                cta_sort_segment<4>(len, src, 0, colidx, perm, s, [&](int t, unsigned long long key) { s[t] = key; });
        } else {
            cta_sort_any(len, src, 0, colidx, perm, s, [&](int t, unsigned long long key) { s[t] = key; });
        }
        __syncthreads();
        for (int t = threadIdx.x; t < len; t += blockDim.x) emit_sorted<E>(s[t], dst + t, src, vals, out_col, out_val);
        __syncthreads();
    }
}

// ---- rows longer than 4096: sorted 4096-key chunks, then merge passes. All
// long rows are cut into tiles of 4096 output positions; every kernel below
// runs one CTA per tile over all long rows at once.
struct LongRow {
    int dst, src, len, pad;
    long long soff;  // offset of the row in the two scratch key buffers
};
struct LongTile {
    int row;    // index into the LongRow table
    int start;  // first position of the tile in the row (multiple of kMedRow)
};

__global__ void long_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                                 const int32_t* __restrict__ inv, const int32_t* __restrict__ out_rowptr,
                                 LongRow* __restrict__ rows)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
        const int i = list[r];
        LongRow lr;
        lr.dst = out_rowptr[i];
        lr.len = out_rowptr[i + 1] - lr.dst;
        lr.src = rowptr[inv[i]];
        lr.pad = 0;
        lr.soff = 0;
        rows[r] = lr;
    }
}

__global__ void __launch_bounds__(256, 2)
    long_chunk_sort_kernel(const LongTile* __restrict__ tiles, int ntiles, const LongRow* __restrict__ rows,
                           const int32_t* __restrict__ colidx, const int32_t* __restrict__ perm,
                           unsigned long long* __restrict__ A)
{
    __shared__ unsigned long long s[kMedRow];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LongTile tl = tiles[t];
        const LongRow R = rows[tl.row];
        const int cl = min(kMedRow, R.len - tl.start);
        unsigned long long* out = A + R.soff + tl.start;
        cta_sort_any(cl, R.src, tl.start, colidx, perm, s, [&](int u, unsigned long long key) { out[u] = key; });
    }
}

// How many of the first d outputs of merging a[0, na) and b[0, nb) come
// from a (keys are unique: the source position breaks column ties).
__device__ __forceinline__ int merge_co_rank(const unsigned long long* a, int na, const unsigned long long* b, int nb,
                                             int d)
{
    int alo = max(0, d - nb), ahi = min(d, na);
    while (alo < ahi) {
        const int am = (alo + ahi) >> 1;
        if (a[am] < b[d - am - 1])
            alo = am + 1;
        else
            ahi = am;
    }
    return alo;
}

// One merge pass: runs of width w are merged pairwise, in[] -> out[]; a
// row whose length is at most 2w is finished by this pass and written
// straight into the output CSR, and a row of at most w was finished by an
// earlier pass and is skipped. Per tile of 4096 outputs, the two input
// ranges it draws from (found by two co-rank searches) are staged in shared
// memory; each thread then merges its 16 consecutive outputs there.
template <typename E>
__global__ void __launch_bounds__(256)
    long_merge_kernel(const LongTile* __restrict__ tiles, int ntiles, const LongRow* __restrict__ rows, int w,
                      const unsigned long long* __restrict__ in, unsigned long long* __restrict__ out,
                      const E* __restrict__ vals, int32_t* __restrict__ out_col, E* __restrict__ out_val)
{
    constexpr int PER = kMedRow / 256;
    __shared__ unsigned long long s_in[kMedRow];
    __shared__ int s_ia[2];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LongTile tl = tiles[t];
        const LongRow R = rows[tl.row];
        if (R.len <= w) continue;  // finished by an earlier pass (uniform over the CTA)
        const bool last = R.len <= 2 * w;
        const int lo = tl.start / (2 * w) * (2 * w);
        const int mid = min(lo + w, R.len), hi = min(lo + 2 * w, R.len);
        const int na = mid - lo, nb = hi - mid;
        const unsigned long long* a = in + R.soff + lo;
        const unsigned long long* b = in + R.soff + mid;
        const int D0 = tl.start - lo, D1 = min(tl.start + kMedRow, R.len) - lo;  // this tile's outputs
        if (threadIdx.x < 2) s_ia[threadIdx.x] = merge_co_rank(a, na, b, nb, threadIdx.x == 0 ? D0 : D1);
        __syncthreads();
        const int ia0 = s_ia[0], ia1 = s_ia[1];
        const int ib0 = D0 - ia0, ib1 = D1 - ia1;
        const int ta = ia1 - ia0, tb = ib1 - ib0;  // ta + tb = D1 - D0 <= kMedRow
        for (int u = threadIdx.x; u < ta + tb; u += blockDim.x) s_in[u] = u < ta ? a[ia0 + u] : b[ib0 + u - ta];
        __syncthreads();
        const int d0 = (int)threadIdx.x * PER, d1 = min(d0 + PER, ta + tb);
        if (d0 < d1) {
            int ia = merge_co_rank(s_in, ta, s_in + ta, tb, d0), ib = d0 - ia;
            for (int d = d0; d < d1; ++d) {
                const bool takeA = ib >= tb || (ia < ta && s_in[ia] < s_in[ta + ib]);
                const unsigned long long key = takeA ? s_in[ia++] : s_in[ta + ib++];
                if (last)
                    emit_sorted<E>(key, R.dst + lo + D0 + d, R.src, vals, out_col, out_val);
                else
                    out[R.soff + lo + D0 + d] = key;
            }
        }
        __syncthreads();  // s_in is reused by the next tile
    }
}

template <typename E>
static int sort_long_rows(const mr_csr_view& A, const int32_t* perm, const int32_t* inv, const int32_t* out_rowptr,
                          int32_t* out_col, E* out_val, const PermStats& hs, const int32_t* large, cudaStream_t st)
{
    const int nl = hs.n_large;
    DevBuf rows_d, tiles_d, scratch;
    MR_TRY(rows_d.alloc(sizeof(LongRow) * (size_t)nl, st));
    long_rows_kernel<<<grid_for(nl, 256), 256, 0, st>>>(large, nl, A.rowptr, inv, out_rowptr, rows_d.as<LongRow>());
    MR_CUDA_TRY(cudaGetLastError());
    std::vector<LongRow> rows((size_t)nl);
    MR_CUDA_TRY(cudaMemcpyAsync(rows.data(), rows_d.p, sizeof(LongRow) * (size_t)nl, cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<LongTile> tiles;
    long long off = 0;
    for (int r = 0; r < nl; ++r) {
        rows[(size_t)r].soff = off;
        off += rows[(size_t)r].len;
        for (int s0 = 0; s0 < rows[(size_t)r].len; s0 += kMedRow) tiles.push_back(LongTile{r, s0});
    }
    const int nt = (int)tiles.size();
    MR_TRY(tiles_d.alloc(sizeof(LongTile) * (size_t)nt, st));
    MR_TRY(scratch.alloc(sizeof(unsigned long long) * 2 * (size_t)off, st));
    // both copies read host vectors that live until the synchronisation below
    MR_CUDA_TRY(cudaMemcpyAsync(rows_d.p, rows.data(), sizeof(LongRow) * (size_t)nl, cudaMemcpyHostToDevice, st));
    MR_CUDA_TRY(cudaMemcpyAsync(tiles_d.p, tiles.data(), sizeof(LongTile) * (size_t)nt, cudaMemcpyHostToDevice, st));
    unsigned long long* bufA = scratch.as<unsigned long long>();
    unsigned long long* bufB = bufA + off;
    const int grid = std::min(nt, sm_count() * 8);
    long_chunk_sort_kernel<<<grid, 256, 0, st>>>(tiles_d.as<LongTile>(), nt, rows_d.as<LongRow>(), A.colidx, perm, bufA);
    MR_CUDA_TRY(cudaGetLastError());
    const E* v = reinterpret_cast<const E*>(A.vals);
    for (int w = kMedRow; w < hs.max_len; w <<= 1) {
        long_merge_kernel<E><<<grid, 256, 0, st>>>(tiles_d.as<LongTile>(), nt, rows_d.as<LongRow>(), w, bufA, bufB, v,
                                                 out_col, out_val);
        MR_CUDA_TRY(cudaGetLastError());
        std::swap(bufA, bufB);
    }
    MR_CUDA_TRY(cudaStreamSynchronize(st));  // the host tables above must outlive their copies
    return MR_OK;
}

template <typename E>
static int launch_sorts(const mr_csr_view& A, const int32_t* perm, const int32_t* inv, const int32_t* out_rowptr,
                        int32_t* out_col, void* out_val, const PermStats& hs, const int32_t* small_list,
                        const int32_t* warp_list, const int32_t* med, const int32_t* large, cudaStream_t st)
{
    const int n = A.n_rows;
    const E* v = reinterpret_cast<const E*>(A.vals);
    E* ov = reinterpret_cast<E*>(out_val);
    sort_tiny_rows_kernel<E><<<grid_for(n, 256), 256, 0, st>>>(n, A.rowptr, A.colidx, v, perm, inv, out_rowptr,
                                                               out_col, ov);
    if (hs.n_small > 0) {
        const int g = (int)std::min<int64_t>(((int64_t)hs.n_small * 32 + 255) / 256, (int64_t)sm_count() * 32);
        sort_small_rows_kernel<E><<<g, 256, 0, st>>>(small_list, hs.n_small, A.rowptr, A.colidx, v, perm, inv,
                                                    out_rowptr, out_col, ov);
    }
    if (hs.n_warp > 0) {
        const int g = (int)std::min<int64_t>(((int64_t)hs.n_warp * 32 + 255) / 256, (int64_t)sm_count() * 32);
        sort_warp_rows_kernel<E><<<g, 256, 0, st>>>(warp_list, hs.n_warp, A.rowptr, A.colidx, v, perm, inv, out_rowptr,
                                                   out_col, ov);
    }
    if (hs.n_med > 0) {
        sort_med_rows_kernel<E, kMedSmall><<<std::min(hs.n_med, sm_count() * 12), 256, 0, st>>>(
            med, hs.n_med, A.rowptr, A.colidx, v, perm, inv, out_rowptr, out_col, ov);
        sort_med_rows_kernel<E, kMedRow><<<std::min(hs.n_med, sm_count() * 8), 256, 0, st>>>(
            med, hs.n_med, A.rowptr, A.colidx, v, perm, inv, out_rowptr, out_col, ov);
    }
    MR_CUDA_TRY(cudaGetLastError());
    if (hs.n_large > 0) MR_TRY(sort_long_rows<E>(A, perm, inv, out_rowptr, out_col, ov, hs, large, st));
    return MR_OK;
}

int permute_csr(const mr_csr_view& A, const int32_t* perm, int32_t* out_rowptr, int32_t* out_colidx, void* out_vals,
                cudaStream_t st)
{
    const int n = A.n_rows;
    if (n == 0) {
        MR_CUDA_TRY(cudaMemsetAsync(out_rowptr, 0, sizeof(int32_t), st));
        return MR_OK;
    }
    DevBuf inv, stats, lists, scan_ws;
    MR_TRY(inv.alloc(sizeof(int32_t) * (size_t)n, st));
    MR_TRY(stats.alloc(sizeof(PermStats), st));
    MR_TRY(lists.alloc(sizeof(int32_t) * 4 * (size_t)n, st));
    MR_TRY(scan_ws.alloc(scan_workspace_bytes(n), st));
    MR_CUDA_TRY(cudaMemsetAsync(stats.p, 0, sizeof(PermStats), st));
    PermStats* ds = stats.as<PermStats>();
    MR_TRY(launch_perm_invert(n, perm, inv.as<int32_t>(), &ds->bad, st));
    MR_TRY(validate_csr_async(A, &ds->bad_csr, st));
    int32_t* small_list = lists.as<int32_t>();
    int32_t* warp_list = small_list + n;
    int32_t* med = warp_list + n;
    int32_t* large = med + n;
    row_lengths_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, A.rowptr, inv.as<int32_t>(), out_rowptr, ds, small_list,
                                                         warp_list, med, large);
    MR_CUDA_TRY(cudaGetLastError());
    MR_TRY(exclusive_scan_i32_ws(out_rowptr, out_rowptr, n, scan_ws.p, st));
    PermStats hs;
    MR_CUDA_TRY(cudaMemcpyAsync(&hs, ds, sizeof(PermStats), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    if (hs.bad_csr) return MR_ERR_INVALID_ARG;
    if (hs.bad) return MR_ERR_INVALID_PERM;
    if (A.dtype == MR_F32)
        return launch_sorts<uint32_t>(A, perm, inv.as<int32_t>(), out_rowptr, out_colidx, out_vals, hs, small_list,
                                      warp_list, med, large, st);
    return launch_sorts<uint16_t>(A, perm, inv.as<int32_t>(), out_rowptr, out_colidx, out_vals, hs, small_list,
                                  warp_list, med, large, st);
}

}  // namespace mr
