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

__global__ void permute_vector_kernel(int n, const int32_t* __restrict__ perm, const float* __restrict__ in,
                                      float* __restrict__ out, int inverse)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = perm[i];
        if (p < 0 || p >= n) continue;
        if (inverse)
            out[i] = in[p];
        else
            out[p] = in[i];
    }
}

int launch_permute_vector(int n, const int32_t* perm, const float* in, float* out, int inverse, cudaStream_t st)
{
    if (n <= 0) return MR_OK;
    permute_vector_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, perm, in, out, inverse);
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

constexpr int kSmallRow = 32;
constexpr int kMedRow = 4096;

struct PermStats {
    int bad;
    int bad_csr;
    int max_len;
    int n_med;
    int n_large;
    unsigned long long large_total;
};

// new row lengths, classification of rows into the medium / large lists
__global__ void row_lengths_kernel(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ inv,
                                   int32_t* __restrict__ len, PermStats* stats, int32_t* __restrict__ med_list,
                                   int32_t* __restrict__ large_list)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = inv[i];
        int l = 0;
        if (o >= 0 && o < n) l = rowptr[o + 1] - rowptr[o];
        len[i] = l;
        if (l > kSmallRow) {
            atomicMax(&stats->max_len, l);
            if (l <= kMedRow) {
                med_list[atomicAdd(&stats->n_med, 1)] = i;
            } else {
                large_list[atomicAdd(&stats->n_large, 1)] = i;
                atomicAdd(&stats->large_total, (unsigned long long)l);
            }
        }
    }
}

template <typename E>
__device__ __forceinline__ void emit_sorted(unsigned long long key, int dst, int src, const E* __restrict__ vals,
                                            int32_t* __restrict__ out_col, E* __restrict__ out_val)
{
    out_col[dst] = (int32_t)(key >> 32);
    out_val[dst] = vals[src + (int)(key & 0xffffffffu)];
}

// rows of length <= 32: one warp per row, bitonic network in registers
template <typename E>
__global__ void __launch_bounds__(256)
    sort_small_rows_kernel(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                           const E* __restrict__ vals, const int32_t* __restrict__ perm,
                           const int32_t* __restrict__ inv, const int32_t* __restrict__ out_rowptr,
                           int32_t* __restrict__ out_col, E* __restrict__ out_val)
{
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        if (len > kSmallRow || len == 0) continue;
        const int src = rowptr[inv[i]];
        unsigned long long key = ~0ull;
        if (lane < len) key = ((unsigned long long)(uint32_t)perm[colidx[src + lane]] << 32) | (unsigned)lane;
        if (len > 1) {
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
        }
        if (lane < len) emit_sorted<E>(key, dst + lane, src, vals, out_col, out_val);
    }
}

// shared-memory bitonic sort of s[0, P) (P a power of two) by one CTA
__device__ void cta_bitonic(unsigned long long* s, int P)
{
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const int i = (t / j) * 2 * j + (t % j);
                const int p = i + j;
                const bool up = (i & k) == 0;
                const unsigned long long a = s[i], b = s[p];
                if ((a > b) == up) {
                    s[i] = b;
                    s[p] = a;
                }
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ int next_pow2(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// rows of length (32, 4096]: one CTA per row (grid-stride over the list)
template <typename E>
__global__ void __launch_bounds__(256)
    sort_med_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                         const int32_t* __restrict__ colidx, const E* __restrict__ vals,
                         const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                         const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                         E* __restrict__ out_val)
{
    __shared__ unsigned long long s[kMedRow];
    for (int r = blockIdx.x; r < count; r += gridDim.x) {
        const int i = list[r];
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        const int src = rowptr[inv[i]];
        const int P = next_pow2(len);
        for (int t = threadIdx.x; t < P; t += blockDim.x)
            s[t] = (t < len) ? (((unsigned long long)(uint32_t)perm[colidx[src + t]] << 32) | (unsigned)t) : ~0ull;
        __syncthreads();
        cta_bitonic(s, P);
        for (int t = threadIdx.x; t < len; t += blockDim.x) emit_sorted<E>(s[t], dst + t, src, vals, out_col, out_val);
        __syncthreads();
    }
}

// rows longer than 4096: sort 4096-key chunks in shared memory, then merge
// runs pairwise through two global scratch buffers (merge-path split per
// thread). One CTA per row.
template <typename E>
__global__ void __launch_bounds__(256)
    sort_large_rows_kernel(const int32_t* __restrict__ list, int count, const int32_t* __restrict__ rowptr,
                           const int32_t* __restrict__ colidx, const E* __restrict__ vals,
                           const int32_t* __restrict__ perm, const int32_t* __restrict__ inv,
                           const int32_t* __restrict__ out_rowptr, int32_t* __restrict__ out_col,
                           E* __restrict__ out_val, unsigned long long* scratch, unsigned long long* scratch_used)
{
    __shared__ unsigned long long s[kMedRow];
    __shared__ unsigned long long s_off;
    for (int r = blockIdx.x; r < count; r += gridDim.x) {
        const int i = list[r];
        const int dst = out_rowptr[i];
        const int len = out_rowptr[i + 1] - dst;
        const int src = rowptr[inv[i]];
        if (threadIdx.x == 0) s_off = atomicAdd(scratch_used, 2ull * (unsigned long long)len);
        __syncthreads();
        unsigned long long* A = scratch + s_off;
        unsigned long long* B = A + len;
        __syncthreads();
        // 1) sorted chunks
        for (int c0 = 0; c0 < len; c0 += kMedRow) {
            const int cl = min(kMedRow, len - c0);
            const int P = next_pow2(cl);
            for (int t = threadIdx.x; t < P; t += blockDim.x)
                s[t] = (t < cl) ? (((unsigned long long)(uint32_t)perm[colidx[src + c0 + t]] << 32) |
                                   (unsigned)(c0 + t))
                                : ~0ull;
            __syncthreads();
            cta_bitonic(s, P);
            for (int t = threadIdx.x; t < cl; t += blockDim.x) A[c0 + t] = s[t];
            __syncthreads();
        }
        // 2) pairwise merges of runs of width w
        for (int w = kMedRow; w < len; w <<= 1) {
            for (int lo = 0; lo < len; lo += 2 * w) {
                const int mid = min(lo + w, len), hi = min(lo + 2 * w, len);
                const int na = mid - lo, nb = hi - mid, tot = na + nb;
                const int per = (tot + blockDim.x - 1) / blockDim.x;
                const int d0 = min((int)threadIdx.x * per, tot), d1 = min(d0 + per, tot);
                // co-rank: a elements taken among the first d0 outputs
                int alo = max(0, d0 - nb), ahi = min(d0, na);
                while (alo < ahi) {
                    const int am = (alo + ahi) >> 1;
                    if (A[lo + am] < A[mid + d0 - am - 1])
                        alo = am + 1;
                    else
                        ahi = am;
                }
                int ia = alo, ib = d0 - alo;
                for (int d = d0; d < d1; ++d) {
                    const bool takeA = ib >= nb || (ia < na && A[lo + ia] < A[mid + ib]);
                    B[lo + d] = takeA ? A[lo + ia++] : A[mid + ib++];
                }
            }
            __syncthreads();
            unsigned long long* t = A;
            A = B;
            B = t;
        }
        for (int t = threadIdx.x; t < len; t += blockDim.x) emit_sorted<E>(A[t], dst + t, src, vals, out_col, out_val);
        __syncthreads();
    }
}

template <typename E>
static int launch_sorts(const mr_csr_view& A, const int32_t* perm, const int32_t* inv, const int32_t* out_rowptr,
                        int32_t* out_col, void* out_val, const PermStats& hs, const int32_t* med, const int32_t* large,
                        cudaStream_t st)
{
    const int n = A.n_rows;
    const E* v = reinterpret_cast<const E*>(A.vals);
    E* ov = reinterpret_cast<E*>(out_val);
    const int grid_small = (int)std::min<int64_t>(((int64_t)n * 32 + 255) / 256, (int64_t)sm_count() * 32);
    sort_small_rows_kernel<E><<<std::max(grid_small, 1), 256, 0, st>>>(n, A.rowptr, A.colidx, v, perm, inv, out_rowptr,
                                                                       out_col, ov);
    if (hs.n_med > 0)
        sort_med_rows_kernel<E><<<std::min(hs.n_med, sm_count() * 8), 256, 0, st>>>(
            med, hs.n_med, A.rowptr, A.colidx, v, perm, inv, out_rowptr, out_col, ov);
    MR_CUDA_TRY(cudaGetLastError());
    if (hs.n_large > 0) {
        DevBuf scratch, used;
        MR_TRY(scratch.alloc(sizeof(unsigned long long) * 2 * (size_t)hs.large_total, st));
        MR_TRY(used.alloc(sizeof(unsigned long long), st));
        MR_CUDA_TRY(cudaMemsetAsync(used.p, 0, sizeof(unsigned long long), st));
        sort_large_rows_kernel<E><<<std::min(hs.n_large, sm_count() * 2), 256, 0, st>>>(
            large, hs.n_large, A.rowptr, A.colidx, v, perm, inv, out_rowptr, out_col, ov,
            scratch.as<unsigned long long>(), used.as<unsigned long long>());
        MR_CUDA_TRY(cudaGetLastError());
    }
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
    MR_TRY(lists.alloc(sizeof(int32_t) * 2 * (size_t)n, st));
    MR_TRY(scan_ws.alloc(scan_workspace_bytes(n), st));
    MR_CUDA_TRY(cudaMemsetAsync(stats.p, 0, sizeof(PermStats), st));
    PermStats* ds = stats.as<PermStats>();
    MR_TRY(launch_perm_invert(n, perm, inv.as<int32_t>(), &ds->bad, st));
    MR_TRY(validate_csr_async(A, &ds->bad_csr, st));
    int32_t* med = lists.as<int32_t>();
    int32_t* large = med + n;
    row_lengths_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, A.rowptr, inv.as<int32_t>(), out_rowptr, ds, med, large);
    MR_CUDA_TRY(cudaGetLastError());
    MR_TRY(exclusive_scan_i32_ws(out_rowptr, out_rowptr, n, scan_ws.p, st));
    PermStats hs;
    MR_CUDA_TRY(cudaMemcpyAsync(&hs, ds, sizeof(PermStats), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    if (hs.bad_csr) return MR_ERR_INVALID_ARG;
    if (hs.bad) return MR_ERR_INVALID_PERM;
    if (A.dtype == MR_F32)
        return launch_sorts<uint32_t>(A, perm, inv.as<int32_t>(), out_rowptr, out_colidx, out_vals, hs, med, large, st);
    return launch_sorts<uint16_t>(A, perm, inv.as<int32_t>(), out_rowptr, out_colidx, out_vals, hs, med, large, st);
}

}  // namespace mr
