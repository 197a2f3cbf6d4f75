// MERBIT merge-path SpMV for sm_100a: plan (descriptor) builder, SpMV kernel
// and the deterministic FP64 carry fix-up.
//
// The plan format is the reference's (include/merbit.cuh:4-20, :55-131): the
// merge of the row-end list (rowptr[1..n]) with the nonzero indices
// 0..nnz-1 is cut into lanes of SIGMA items and tiles of 32 lanes. Per lane a
// descriptor word packs the row-end flags of its SIGMA items, its row offset
// and its nonzero offset from the tile start; per tile tile_x = first
// nonzero, tile_y = first row (bit 31: the tile lies inside one row).
//
// B200 design (own code, not the reference's kernel):
//  * plan: one CTA stages the rowptr window its 256 lanes can touch into
//    shared memory, then every lane runs its merge-path search and its
//    SIGMA-step walk out of shared memory (the reference walks global rowptr).
//  * SpMV: one warp per tile. The tile's colidx/values are streamed with
//    16-byte evict-first loads, x is gathered with an L2 evict-last policy,
//    products are staged in shared memory; each lane walks its SIGMA items
//    from its descriptor, keeping finished rows in registers; a warp
//    segmented scan (shuffles) carries partial sums across lanes; finished
//    rows leave through shared memory as coalesced stores. No atomics: the
//    partial sum of the row still open at the tile end goes to a per-tile
//    carry slot, and a second kernel adds each run of carries to its row in
//    FP64 in tile order. Results are bitwise reproducible run to run.
#include <algorithm>

#include "common.cuh"
#include "internal.hpp"

namespace mr {

// ----------------------------------------------------------------- plan ----

// Merge-path search along cross diagonal `diag`: the number of rows already
// ended (cy) and nonzeros consumed (cx), with cy searched in [lo, hi].
// off(i) returns rowptr[i]. Same decision rule as merge_search
// (include/merbit.cuh:24-53), so the same unique path point.
template <typename Off>
__device__ __forceinline__ void merge_path_search(Off off, int nnz, int nrow, int diag, int lo, int hi,
                                                  int& cx, int& cy)
{
    int ymin = max(max(diag - nnz, 0), lo);
    int ymax = min(min(diag, nrow), hi);
    while (ymin < ymax) {
        int mid = (ymin + ymax) >> 1;
        if (off(mid + 1) <= diag - mid - 1)
            ymin = mid + 1;
        else
            ymax = mid;
    }
    cx = diag - ymin;
    cy = min(ymin, nrow);
}

constexpr int kPlanBlock = 256;

template <typename Desc>
__global__ void __launch_bounds__(kPlanBlock)
    merbit_plan_kernel(const int* __restrict__ rowptr, int nrow, int nnz, int sigma, int lane_num, int tile_num,
                       uint32_t* __restrict__ tile_x, uint32_t* __restrict__ tile_y, Desc* __restrict__ lane_desc)
{
    extern __shared__ int s_off[];  // rowptr[r0 .. r0 + cnt)
    __shared__ int s_r0, s_cnt;
    constexpr bool wide = sizeof(Desc) == 8;
    constexpr int sh_flag = wide ? 22 : 18;
    constexpr int sh_dy = wide ? 11 : 9;

    const int64_t items = (int64_t)nnz + nrow;
    const int lane0 = blockIdx.x * kPlanBlock;
    const int gid = lane0 + threadIdx.x;
    if (threadIdx.x == 0) {
        auto goff = [&](int i) { return __ldg(rowptr + i); };
        int cx, ya, yb;
        int d0 = (int)min64((int64_t)lane0 * sigma, items);
        int d1 = (int)min64((int64_t)(lane0 + kPlanBlock) * sigma, items);
        merge_path_search(goff, nnz, nrow, d0, 0, nrow, cx, ya);
        merge_path_search(goff, nnz, nrow, d1, ya, nrow, cx, yb);
        s_r0 = ya;
        s_cnt = min(yb + 2, nrow + 1) - ya;  // rowptr[ya .. min(yb + 1, nrow)]
    }
    __syncthreads();
    const int r0 = s_r0, cnt = s_cnt;
    for (int i = threadIdx.x; i < cnt; i += kPlanBlock) s_off[i] = __ldg(rowptr + r0 + i);
    __syncthreads();

    if (gid < lane_num) {
        const int tile = gid >> 5, lid = threadIdx.x & 31;
        const int warp_len = ((tile + 1) * 32 < lane_num) ? 32 : (lane_num - tile * 32);
        const unsigned mask = (warp_len == 32) ? 0xffffffffu : ((1u << warp_len) - 1u);
        const int lane_items = (int)min64((int64_t)sigma, items - (int64_t)gid * sigma);
        // clamp keeps a malformed rowptr from reading past the staged window
        auto soff = [&](int i) { return s_off[min(max(i - r0, 0), cnt - 1)]; };
        int cx, cy;
        merge_path_search(soff, nnz, nrow, gid * sigma, r0, r0 + cnt - 1, cx, cy);
        const int wx = __shfl_sync(mask, cx, 0);
        const int wy = __shfl_sync(mask, cy, 0);
        const Desc dx = (Desc)(uint32_t)(cx - wx);
        const Desc dy = (Desc)(uint32_t)(cy - wy);
        const int y_start = cy;
        Desc flags = 0;
        for (int i = 0; i < lane_items; ++i) {
            if (cx < soff(cy + 1)) {
                ++cx;
            } else {
                flags |= (Desc)1 << i;
                ++cy;
            }
        }
        lane_desc[gid] = (flags << sh_flag) | (dy << sh_dy) | dx;
        const bool single_row = __all_sync(mask, y_start == cy);
        if (lid == 0) {
            tile_x[tile] = (uint32_t)wx;
            tile_y[tile] = (single_row ? 0x80000000u : 0u) | (uint32_t)wy;
        }
    } else if (gid == lane_num) {
        tile_x[tile_num] = (uint32_t)nnz;
        tile_y[tile_num] = (uint32_t)nrow;
    }
}

int launch_merbit_plan(const int* rowptr, int nrow, int nnz, int sigma, int lane_num, int tile_num,
                       uint32_t* tile_x, uint32_t* tile_y, void* lane_desc, cudaStream_t st)
{
    const int grid = lane_num / kPlanBlock + 1;  // one extra thread writes the sentinel
    const size_t smem = sizeof(int) * ((size_t)kPlanBlock * sigma + 2);
    if (sigma < 15) {
        if (smem > 48 * 1024)
            MR_CUDA_TRY(cudaFuncSetAttribute(merbit_plan_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        merbit_plan_kernel<uint32_t><<<grid, kPlanBlock, smem, st>>>(rowptr, nrow, nnz, sigma, lane_num, tile_num,
                                                                     tile_x, tile_y, (uint32_t*)lane_desc);
    } else {
        if (smem > 48 * 1024)
            MR_CUDA_TRY(cudaFuncSetAttribute(merbit_plan_kernel<unsigned long long>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        merbit_plan_kernel<unsigned long long><<<grid, kPlanBlock, smem, st>>>(
            rowptr, nrow, nnz, sigma, lane_num, tile_num, tile_x, tile_y, (unsigned long long*)lane_desc);
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

// ----------------------------------------------------------------- SpMV ----

template <int SIGMA> struct DescOf {
    using T = typename std::conditional<(SIGMA < 15), uint32_t, unsigned long long>::type;
    static constexpr int sh_flag = SIGMA < 15 ? 18 : 22;
    static constexpr int sh_dy = SIGMA < 15 ? 9 : 11;
    static constexpr unsigned mask_d = SIGMA < 15 ? 0x1ffu : 0x7ffu;
};

// Shared-memory words per warp: products of one tile (<= 32*SIGMA), shifted
// by up to 3 so that 16-byte vectors stay aligned, plus slack.
template <int SIGMA> constexpr int tile_smem_words() { return 32 * SIGMA + 8; }

template <typename V, int SIGMA, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    merbit_spmv_kernel(const uint32_t* __restrict__ tile_x, const uint32_t* __restrict__ tile_y,
                       const typename DescOf<SIGMA>::T* __restrict__ lane_desc, int tile_num, int lane_num,
                       int64_t items, const int* __restrict__ colidx, const V* __restrict__ vals, int nnz,
                       const float* __restrict__ x, float* __restrict__ y, float* __restrict__ carry, int vec_ok)
{
    using D = DescOf<SIGMA>;
    using DT = typename D::T;
    constexpr int TW = tile_smem_words<SIGMA>();
    __shared__ __align__(16) float s_buf[WARPS][TW];

    const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
    const int tile = blockIdx.x * WARPS + warp;
    if (tile >= tile_num) return;
    float* s = s_buf[warp];
    const uint64_t pol = l2_evict_last_policy();

    const int x0 = (int)__ldg(tile_x + tile);
    const int x1 = (int)__ldg(tile_x + tile + 1);
    const uint32_t ty0 = __ldg(tile_y + tile);
    const int y0 = (int)(ty0 & 0x7fffffffu);
    const int y1 = (int)(__ldg(tile_y + tile + 1) & 0x7fffffffu);
    const bool single_row = (ty0 >> 31) != 0;

    // ---- stage products vals[k] * x[colidx[k]] for k in [x0, x1) ---------
    const int a0 = x0 & ~3;           // 16-byte aligned start
    const int shift = x0 - a0;        // products of x0 land at s[shift]
    const int nvec = (x1 - a0 + 3) >> 2;
    float part = 0.f;                 // single-row tiles: running dot product
    for (int v = lid; v < nvec; v += 32) {
        const int k = a0 + 4 * v;
        float p[4];
        if (vec_ok && k + 3 < nnz) {
            const int4 c = ld_stream(reinterpret_cast<const int4*>(colidx + k));
            float w[4];
            Vec4<V>::unpack(ld_stream(reinterpret_cast<const typename Vec4<V>::T*>(vals + k)), w);
            const int cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) p[j] = (k + j >= x0 && k + j < x1) ? w[j] * ld_x(x + cc[j], pol) : 0.f;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int kk = k + j;
                p[j] = (kk >= x0 && kk < x1)
                           ? ValueTraits<V>::f(ld_stream(vals + kk)) * ld_x(x + ld_stream(colidx + kk), pol)
                           : 0.f;
            }
        }
        if (single_row) {
            part += (p[0] + p[1]) + (p[2] + p[3]);
        } else {
            *reinterpret_cast<float4*>(s + 4 * v) = make_float4(p[0], p[1], p[2], p[3]);
        }
    }
    if (single_row) {
        // every item of this tile is a nonzero of row y0 (== y1): the whole
        // tile is a carry into that row
        part = warp_sum(part);
        if (lid == 0) carry[tile] = part;
        return;
    }
    __syncwarp();

    // ---- walk this lane's SIGMA merge items -------------------------------
    const int gid = tile * 32 + lid;
    int lane_items = 0;
    DT d = 0;
    if (gid < lane_num) {
        lane_items = (int)min64((int64_t)SIGMA, items - (int64_t)gid * SIGMA);
        d = __ldg(lane_desc + gid);
    }
    const uint32_t flags = (uint32_t)(d >> D::sh_flag) & ((lane_items >= 32) ? 0xffffffffu : ((1u << lane_items) - 1u));
    int xi = shift + (int)(d & D::mask_d);
    const int dy = (int)((d >> D::sh_dy) & D::mask_d);

    float rows[SIGMA];  // finished row sums, indexed by the item that ends them
    float cur = 0.f, head = 0.f;
#pragma unroll
    for (int i = 0; i < SIGMA; ++i) {
        rows[i] = 0.f;
        if (i < lane_items) {
            if ((flags >> i) & 1u) {
                rows[i] = cur;
                cur = 0.f;
            } else {
                cur += s[xi];
                ++xi;
            }
        }
    }
    const int nflags = __popc(flags);
    const int first = nflags ? (__ffs(flags) - 1) : SIGMA;
#pragma unroll
    for (int i = 0; i < SIGMA; ++i)
        if (i == first) head = rows[i];

    // ---- warp segmented scan of the carried partial sums ------------------
    // value: what this lane passes on (sum after its last row end); a lane
    // with a row end starts a new segment.
    float incl = cur;
    bool seg = nflags != 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float nv = __shfl_up_sync(0xffffffffu, incl, o);
        const bool ns = __shfl_up_sync(0xffffffffu, seg, o);
        if (lid >= o && !seg) {
            incl += nv;
            seg = ns;
        }
    }
    float carry_in = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lid == 0) carry_in = 0.f;
    const float tile_carry = __shfl_sync(0xffffffffu, incl, 31);
    head += carry_in;
    __syncwarp();  // all lanes are done reading products

    // ---- finished rows -> shared -> coalesced stores ----------------------
    int r = dy;
#pragma unroll
    for (int i = 0; i < SIGMA; ++i) {
        if ((flags >> i) & 1u) {
            s[r] = (i == first) ? head : rows[i];
            ++r;
        }
    }
    __syncwarp();
    const int nrows = y1 - y0;
    for (int j = lid; j < nrows; j += 32) __stcs(y + y0 + j, s[j]);
    if (lid == 0) carry[tile] = tile_carry;
}

// One thread per run of consecutive tiles whose open row at the tile end is
// the same row R: y[R] += sum of their carries, summed in FP64 in tile order.
__global__ void merbit_fixup_kernel(const uint32_t* __restrict__ tile_y, const float* __restrict__ carry,
                                    int tile_num, int nrow, float* __restrict__ y)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tile_num) return;
    const int R = (int)(__ldg(tile_y + t + 1) & 0x7fffffffu);
    if (R >= nrow) return;
    if (t > 0 && (int)(__ldg(tile_y + t) & 0x7fffffffu) == R) return;  // not the first tile of the run
    double s = 0.0;
    int u = t;
    do {
        s += (double)carry[u];
        ++u;
    } while (u < tile_num && (int)(__ldg(tile_y + u + 1) & 0x7fffffffu) == R);
    y[R] = (float)((double)y[R] + s);
}

template <typename V, int SIGMA, int WARPS>
static int launch_spmv_t(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x, float* y,
                         float* carry, cudaStream_t st)
{
    const int grid = (p.tile_num + WARPS - 1) / WARPS;
    const int vec_ok = ((reinterpret_cast<uintptr_t>(colidx) & 15) == 0) &&
                       ((reinterpret_cast<uintptr_t>(vals) & (4 * sizeof(V) - 1)) == 0);
    if (grid > 0)
        merbit_spmv_kernel<V, SIGMA, WARPS><<<grid, WARPS * 32, 0, st>>>(
            p.tile_x, p.tile_y, reinterpret_cast<const typename DescOf<SIGMA>::T*>(p.lane_desc), p.tile_num,
            p.lane_num, (int64_t)p.n_rows + p.nnz, colidx, reinterpret_cast<const V*>(vals), nnz, x, y, carry,
            vec_ok);
    MR_CUDA_TRY(cudaGetLastError());
    if (p.tile_num > 0) {
        merbit_fixup_kernel<<<(p.tile_num + 255) / 256, 256, 0, st>>>(p.tile_y, carry, p.tile_num, p.n_rows, y);
        MR_CUDA_TRY(cudaGetLastError());
    }
    return MR_OK;
}

template <typename V, int SIGMA>
static int launch_spmv_w(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x, float* y,
                         float* carry, cudaStream_t st)
{
    switch (p.block) {
    case 128: return launch_spmv_t<V, SIGMA, 4>(p, colidx, vals, nnz, x, y, carry, st);
    case 512:
        // 16 warps only while the static staging buffers fit in 48 KB
        if constexpr (16 * tile_smem_words<SIGMA>() * 4 <= 48 * 1024)
            return launch_spmv_t<V, SIGMA, 16>(p, colidx, vals, nnz, x, y, carry, st);
        else
            return launch_spmv_t<V, SIGMA, 8>(p, colidx, vals, nnz, x, y, carry, st);
    default: return launch_spmv_t<V, SIGMA, 8>(p, colidx, vals, nnz, x, y, carry, st);
    }
}

template <typename V>
static int launch_spmv_v(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x, float* y,
                         float* carry, cudaStream_t st)
{
    switch (p.sigma) {
#define MR_SIGMA_CASE(S) \
    case S: return launch_spmv_w<V, S>(p, colidx, vals, nnz, x, y, carry, st);
        MR_SIGMA_CASE(7)
        MR_SIGMA_CASE(10)
        MR_SIGMA_CASE(14)
        MR_SIGMA_CASE(16)
        MR_SIGMA_CASE(20)
        MR_SIGMA_CASE(24)
        MR_SIGMA_CASE(28)
        MR_SIGMA_CASE(32)
#undef MR_SIGMA_CASE
    default: return MR_ERR_UNSUPPORTED;
    }
}

bool merbit_sigma_supported(int sigma)
{
    switch (sigma) {
    case 7: case 10: case 14: case 16: case 20: case 24: case 28: case 32: return true;
    default: return false;
    }
}

int launch_merbit_spmv(const MerbitPlan& p, const int* colidx, const void* vals, int dtype, const float* x, float* y,
                       float* carry, cudaStream_t st)
{
    const int nnz = (int)p.nnz;
    switch (dtype) {
    case MR_F32: return launch_spmv_v<float>(p, colidx, vals, nnz, x, y, carry, st);
    case MR_F16: return launch_spmv_v<__half>(p, colidx, vals, nnz, x, y, carry, st);
    case MR_BF16: return launch_spmv_v<__nv_bfloat16>(p, colidx, vals, nnz, x, y, carry, st);
    default: return MR_ERR_UNSUPPORTED;
    }
}

}  // namespace mr
