// pGOrder on the GPU: the gorder4 ordering (GRAPH::gorder4 / order_on_cpu,
// src/class.cu:2608-2690, :2220-2314) with one warp per block of vsize
// vertex ids, bit-identical to the host ordering (csrc/pgorder.cpp) and so
// to the reference.
//
// Each block's ordering is a sequential greedy over a bucket queue whose link
// order decides ties (Integer_Heap, include/integer_heap.cuh:34-151), so the
// queue operations must happen in the host's order. Per block, one warp:
//  * the queue lives in shared memory (16-bit links and keys: a key never
//    exceeds width * (L - 1) + 1, since each of the `width` vertices of the
//    window adds at most one per column of its row and rows of L or more
//    entries add nothing);
//  * for every placed vertex, the columns of its row are visited 32 at a
//    time, one per lane: each lane counts the still-queued vertices of the
//    block in its column, a warp prefix sum gives every column its slot in a
//    shared-memory hit list, the lanes write their hits in entry order, and
//    lane 0 applies the modifies in that (column, entry) order, exactly as
//    the host loop does (a chunk with more hits than the list holds is
//    walked column by column instead, same order);
//  * pops, the seed choice and the window decrements follow the host code.
// The column lists (rows ascending within a column, the reference's
// sort(true) + coo2csr) come from a stable radix sort of (column, row).
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

constexpr int kHitCap = 4096;  // hit-list entries per block (int16)

struct Queue16 {
    int16_t* left;
    int16_t* right;
    int16_t* key1;  // bucket the vertex sits in
    int16_t* key2;  // pending change
    int16_t* htab;  // bucket heads, -1 = empty
    int htab_len;
    int* err;       // set when a key leaves [0, htab_len) (matrices with repeated entries)
    int pmax, cnt;

    __device__ void remove(int v)
    {
        int16_t& head = htab[key1[v]];
        const int l = left[v], r = right[v];
        if (head == v) {
            if (r == v) {
                head = -1;
                return;
            }
            head = (int16_t)r;
        }
        right[l] = (int16_t)r;
        left[r] = (int16_t)l;
        left[v] = (int16_t)v;
        right[v] = (int16_t)v;
    }
    __device__ void insert(int v)
    {
        int k = key1[v] + key2[v];
        if ((unsigned)k >= (unsigned)htab_len) {  // result no longer valid; keep every access in bounds
            *err = 1;
            k = k < 0 ? 0 : htab_len - 1;
        }
        key1[v] = (int16_t)k;
        key2[v] = 0;
        int16_t& head = htab[k];
        if (head < 0) {
            head = (int16_t)v;
        } else {
            const int h = head, hr = right[h];
            left[v] = (int16_t)h;
            right[v] = (int16_t)hr;
            left[hr] = (int16_t)v;
            right[h] = (int16_t)v;
        }
    }
    __device__ void modify(int v, int d)
    {
        key2[v] = (int16_t)(key2[v] + d);
        if (key2[v] > 0) {
            remove(v);
            insert(v);
            if (key1[v] > pmax) pmax = key1[v];
        }
    }
    __device__ int pop()
    {
        while (cnt > 0) {
            while (pmax > 0 && htab[pmax] < 0) --pmax;
            int t = htab[pmax];
            while (t >= 0) {
                if (key2[t] == 0) {
                    remove(t);
                    --cnt;
                    return t;
                }
                remove(t);
                insert(t);
                t = htab[pmax];
            }
        }
        return -1;
    }
};

// One warp per block of vertex ids [start, start + len).
__global__ void __launch_bounds__(32)
    pgorder_block_kernel(int n, int vsize, int width, int degree, const int32_t* __restrict__ roff,
                         const int32_t* __restrict__ rind, const int32_t* __restrict__ coff,
                         const int32_t* __restrict__ cind, int htab_len, uint32_t* __restrict__ perm, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x;
    const int start = blockIdx.x * vsize;
    const int len = min(vsize, n - start);
    int16_t* left = reinterpret_cast<int16_t*>(smem);
    int16_t* right = left + vsize;
    int16_t* key1 = right + vsize;
    int16_t* key2 = key1 + vsize;
    int16_t* htab = key2 + vsize;
    uint32_t* sts = reinterpret_cast<uint32_t*>(htab + ((htab_len + 1) & ~1));  // 1 = still queued
    int16_t* hits = reinterpret_cast<int16_t*>(sts + (vsize + 31) / 32);
    for (int i = lane; i < len; i += 32) {
        key1[i] = 0;
        key2[i] = 0;
    }
    for (int i = lane; i < htab_len; i += 32) htab[i] = -1;
    for (int i = lane; i < (len + 31) / 32; i += 32) sts[i] = 0xffffffffu;
    // seed: the largest column count, the first one on ties
    int best = -1, bid = 0;
    for (int i = lane; i < len; i += 32) {
        const int d = coff[start + i + 1] - coff[start + i];
        if (d > best) {
            best = d;
            bid = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int ob = __shfl_xor_sync(0xffffffffu, best, o), oi = __shfl_xor_sync(0xffffffffu, bid, o);
        if (ob > best || (ob == best && oi < bid)) {
            best = ob;
            bid = oi;
        }
    }
    __syncwarp();
    Queue16 q{left, right, key1, key2, htab, htab_len, err, 0, 0};
    if (lane == 0) {
        // all block vertices enter bucket 0 in id order, then the seed gains one
        for (int i = 0; i < len; ++i) {
            left[i] = (int16_t)i;
            right[i] = (int16_t)i;
            q.insert(i);
        }
        q.cnt = len;
        q.modify(bid, 1);
    }
    auto queued = [&](int k) -> int {  // block-local vertex of column entry k if still queued, else -1
        const unsigned ww = (unsigned)(__ldg(cind + k) - start);
        return (ww < (unsigned)len && ((sts[ww >> 5] >> (ww & 31)) & 1u)) ? (int)ww : -1;
    };
    // one bump pass: the vertices sharing a column with u gain d
    auto bump = [&](int u, int d) {
        const int rb = __ldg(roff + u), re = __ldg(roff + u + 1);
        if (re - rb >= degree) return;
        for (int j0 = rb; j0 < re; j0 += 32) {
            const int j = j0 + lane;
            int cb = 0, ce = 0;
            if (j < re) {
                const int c = __ldg(rind + j);
                cb = __ldg(coff + c);
                ce = __ldg(coff + c + 1);
                if (ce - cb >= degree) ce = cb;  // columns of L or more entries add nothing
            }
            int cnt = 0;
#pragma unroll 8
            for (int k = cb; k < ce; ++k) cnt += queued(k) >= 0;  // independent loads: several in flight
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            if (total == 0) continue;
            if (total <= kHitCap) {
                int p = incl - cnt;
                for (int k = cb; k < ce && p < incl; ++k) {
                    const int w = queued(k);
                    if (w >= 0) hits[p++] = (int16_t)w;
                }
                __syncwarp();
                if (lane == 0)
                    for (int i = 0; i < total; ++i) q.modify(hits[i], d);
                __syncwarp();
            } else {
                // too many hits for the list: column by column, same order
                const int nj = min(32, re - j0);
                for (int t = 0; t < nj; ++t) {
                    const int b = __shfl_sync(0xffffffffu, cb, t), e = __shfl_sync(0xffffffffu, ce, t);
                    for (int k0 = b; k0 < e; k0 += 32) {
                        const int w = k0 + lane < e ? queued(k0 + lane) : -1;
                        unsigned m = __ballot_sync(0xffffffffu, w >= 0);
                        while (m) {
                            const int l = __ffs(m) - 1;
                            const int wv = __shfl_sync(0xffffffffu, w, l);
                            if (lane == 0) q.modify(wv, d);
                            m &= m - 1;
                        }
                    }
                }
            }
        }
    };
    for (int pos = 0; pos < len; ++pos) {
        int u = 0;
        if (lane == 0) {
            u = q.pop();
            if (u < 0) {  // cannot happen with a consistent queue; flagged, and kept in bounds
                *err = 1;
                u = 0;
            }
            sts[u >> 5] &= ~(1u << (u & 31));
            perm[start + pos] = (uint32_t)(u + start);
        }
        u = __shfl_sync(0xffffffffu, u, 0);
        __syncwarp();
        bump(u + start, 1);
        if (pos >= width) {
            const int old = (int)perm[start + pos - width];  // written by lane 0 of this warp
            bump(old, -1);
        }
        __syncwarp();
    }
}

__global__ void iota_u32_kernel(int32_t* __restrict__ a, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void row_of_kernel(const int32_t* __restrict__ rowptr, int n, int32_t* __restrict__ row)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) row[k] = r;
}

__global__ void col_count_kernel(const uint32_t* __restrict__ sorted_cols, int nnz, int n, int32_t* __restrict__ coff)
{
    // coff[c] = first position of column c in the sorted list (lower bound)
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= n; c += gridDim.x * blockDim.x) {
        int lo = 0, hi = nnz;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)sorted_cols[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        coff[c] = lo;
    }
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8)); }

}  // namespace

int pgorder_gpu(int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t nnz, int32_t vsize, int32_t width,
                uint32_t* perm, cudaStream_t st)
{
    if (n == 0) return MR_OK;
    if (vsize <= 0) vsize = pgorder_width(n, nnz);
    const int degree = (int)(std::sqrt((double)n) / 4);
    const long long htab_len = (long long)width * std::max(degree - 1, 0) + 2;
    if (vsize > 32767 || htab_len > 32767) return MR_ERR_UNSUPPORTED;
    const size_t smem = sizeof(int16_t) * (4 * (size_t)vsize + (size_t)((htab_len + 1) & ~1LL)) +
                        sizeof(uint32_t) * (size_t)((vsize + 31) / 32) + sizeof(int16_t) * kHitCap;
    int optin = 0, dev = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > (size_t)optin) return MR_ERR_UNSUPPORTED;
    // column lists: stable sort of (column, row) pairs in row order
    {
        // column indices index the offset array directly: check them first
        const mr_csr_view A{n, n, nnz, rowptr, colidx, colidx, MR_F32};
        int ok = 0;
        MR_TRY(validate_csr(A, &ok, st));
        if (!ok) return MR_ERR_INVALID_ARG;
    }
    DevBuf k0, k1, v0, v1, coff, err;
    MR_TRY(err.alloc(sizeof(int), st));
    MR_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    const size_t m = (size_t)std::max(nnz, 1);
    MR_TRY(k0.alloc(sizeof(uint32_t) * m, st));
    MR_TRY(k1.alloc(sizeof(uint32_t) * m, st));
    MR_TRY(v0.alloc(sizeof(int32_t) * m, st));
    MR_TRY(v1.alloc(sizeof(int32_t) * m, st));
    MR_TRY(coff.alloc(sizeof(int32_t) * ((size_t)n + 1), st));
    if (nnz > 0) {
        MR_CUDA_TRY(cudaMemcpyAsync(k0.p, colidx, sizeof(int32_t) * (size_t)nnz, cudaMemcpyDeviceToDevice, st));
        row_of_kernel<<<grid_n(n), 256, 0, st>>>(rowptr, n, v0.as<int32_t>());
        int bits = 1;
        while (bits < 31 && (1 << bits) < n) ++bits;
        uint32_t* keys = k0.as<uint32_t>();
        int32_t* rows = v0.as<int32_t>();
        MR_TRY(radix_sort_pairs_u32(keys, rows, k1.as<uint32_t>(), v1.as<int32_t>(), nnz, bits, st));
        col_count_kernel<<<grid_n((int64_t)n + 1), 256, 0, st>>>(keys, nnz, n, coff.as<int32_t>());
        MR_CUDA_TRY(cudaGetLastError());
        const int nb = (int)(((int64_t)n + vsize - 1) / vsize);
        MR_CUDA_TRY(cudaFuncSetAttribute(pgorder_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pgorder_block_kernel<<<nb, 32, smem, st>>>(n, vsize, width, degree, rowptr, colidx, coff.as<int32_t>(), rows,
                                                   (int)htab_len, perm, err.as<int>());
        MR_CUDA_TRY(cudaGetLastError());
        int h = 0;
        MR_CUDA_TRY(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MR_CUDA_TRY(cudaStreamSynchronize(st));
        if (h) return MR_ERR_UNSUPPORTED;  // keys beyond the table: use the host ordering
    } else {
        iota_u32_kernel<<<grid_n(n), 256, 0, st>>>(reinterpret_cast<int32_t*>(perm), n);
        MR_CUDA_TRY(cudaGetLastError());
    }
    MR_CUDA_TRY(cudaStreamSynchronize(st));  // scratch released on return
    return MR_OK;
}

}  // namespace mr
