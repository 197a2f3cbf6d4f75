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
//  * persistent form (block 1024): one CTA per SM over a chunk of tiles cut
//    at plan time by estimated cost, with the hub cache of the hottest x
//    columns in shared memory and the carry fix-up fused (runs inside a
//    chunk walked in shared memory, runs across chunk starts finished from
//    a plan-time table by the later of the two neighbouring CTAs): one
//    launch per SpMV, bit-identical to the two-kernel form.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.hpp"
#include "merbit_tile.cuh"

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

template <typename V, int SIGMA, int WARPS, int GM>
__global__ void __launch_bounds__(WARPS * 32) merbit_spmv_kernel(const MerbitOperand<V, SIGMA> m, int tile_num)
{
    __shared__ __align__(16) float s_buf[WARPS][tile_smem_words<SIGMA>()];
    // the fix-up grid (launched as a programmatic dependent) may be
    // scheduled once every CTA of this grid has started; it waits for this
    // grid's completion before it reads a carry
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int warp = threadIdx.x >> 5;
    const int tile = blockIdx.x * WARPS + warp;
    if (tile >= tile_num) return;
    // matrix streams bypass L1 and are evict-first in L2, so L1 and L2 keep
    // x (0.2719 vs 0.2737 ms at R-MAT s22, SIGMA 14, 256 threads)
    merbit_tile<V, SIGMA, true, false, GM>(m, tile, s_buf[warp],
                                          TilePolicy{l2_evict_last_policy(), l2_evict_first_policy()});
}

// ---- persistent form: one CTA of 32 warps per SM sweeps a contiguous chunk
// of tiles, so the warps resident on an SM work on neighbouring rows and the
// reordered matrix's x reuse is caught by L1 (the streams bypass L1). The
// chunk bounds come from the plan, balanced by estimated cost (a tile's x
// gathers that miss the hub cache dominate its time, so equal tile counts
// leave some SMs working 20% longer than the mean), or are equal tile counts
// when the plan has none. Carry runs that stay inside a chunk are finished
// by the chunk's CTA after a barrier, walked in shared memory. A run that
// crosses a chunk start is finished, from the plan's run table, by the
// second of the two CTAs beside that start to get there (arrival counters,
// no waiting), or, when it starts before the previous chunk, by the last CTA
// to finish (atomic ticket after a fence); plans without a table leave
// every crossing run to the last CTA. Same FP64 run sums, same order, as the
// two-kernel form: the results are bit-identical.
//
// Inside a chunk the warps take the first three quarters of the tiles round
// robin (warp w: tiles w, w + 32, ...; the 32 warps stay on 32 adjacent
// tiles) and the rest one at a time from a shared-memory counter, so that
// warps whose tiles were cheap take more of the tail instead of waiting at the
// barrier for the slowest (tile costs vary ~30%; a fully counter-driven loop
// is slower). Which warp runs a tile does not change its result.
constexpr int kPersistWarps = 32;
constexpr int kStaticNum = 3, kStaticDen = 4;

__device__ __forceinline__ int open_row(const uint32_t* tile_y, int t) { return tile_open_row(tile_y, t); }

// run that starts in [t0, t1) and whose row ends inside the chunk
__device__ __forceinline__ void fixup_in_chunk(const uint32_t* __restrict__ tile_y, const float* carry, int t0, int t1,
                                               int nrow, float* y, int t)
{
    const int R = open_row(tile_y, t);
    if (R >= nrow) return;
    if (t > 0 && open_row(tile_y, t - 1) == R) return;  // not the first tile of its run
    double acc = 0.0;
    int u = t;
    while (u < t1 && open_row(tile_y, u) == R) {
        acc += (double)carry[u];
        ++u;
    }
    if (u >= t1) return;  // the row ends in a later chunk: boundary pass
    y[R] = (float)((double)y[R] + acc);
}

// Run that crosses the boundary b at the start of a chunk [b, e) and whose
// row ends inside that chunk (each crossing run is finished at exactly one
// boundary; an empty chunk finishes none), for one warp: the run's ends are
// found 32 tiles per step with ballots (open rows never decrease along the
// tiles, so a run is contiguous), and its carries are summed in FP64 in tile
// order, as in fixup_in_chunk.
__device__ __forceinline__ void fixup_boundary_warp(const uint32_t* __restrict__ tile_y, const float* carry,
                                                    int tile_num, int b, int e, int nrow, float* y, int lane)
{
    if (b <= 0 || b >= tile_num) return;
    const int p = b - 1;
    const int R = open_row(tile_y, p);
    if (R >= nrow) return;
    int ue = p;  // last tile of the run
    for (;;) {
        const int q = ue + 1 + lane;
        const unsigned m = __ballot_sync(0xffffffffu, q < tile_num && open_row(tile_y, q) == R);
        if (m != 0xffffffffu) {
            ue += __ffs(~m) - 1;
            break;
        }
        ue += 32;
    }
    if (ue + 1 >= e) return;  // ends beyond this chunk
    int u0 = p;  // first tile of the run
    for (;;) {
        const int q = u0 - 1 - lane;
        const unsigned m = __ballot_sync(0xffffffffu, q >= 0 && open_row(tile_y, q) == R);
        if (m != 0xffffffffu) {
            u0 -= __ffs(~m) - 1;
            break;
        }
        u0 -= 32;
    }
    double acc = 0.0;
    for (int base = u0; base <= ue; base += 32) {
        const float c = base + lane <= ue ? __ldcg(carry + base + lane) : 0.f;
        const int cnt = min(32, ue - base + 1);
        for (int j = 0; j < cnt; ++j) acc += (double)__shfl_sync(0xffffffffu, c, j);
    }
    if (lane == 0) y[R] = (float)((double)__ldcg(y + R) + acc);
}

// Finishes a carry run known from the plan: carries of tiles u0 .. ue summed
// in FP64 in tile order and added to y[R] (one warp).
__device__ __forceinline__ void finish_run(const int4 run, const float* carry, float* y, int lane)
{
    const int R = run.x, u0 = run.y, ue = run.z;
    const float yr = lane == 0 ? __ldcg(y + R) : 0.f;
    double acc = 0.0;
    for (int base = u0; base <= ue; base += 32) {
        const float c = base + lane <= ue ? __ldcg(carry + base + lane) : 0.f;
        const int cnt = min(32, ue - base + 1);
        for (int j = 0; j < cnt; ++j) acc += (double)__shfl_sync(0xffffffffu, c, j);
    }
    if (lane == 0) y[R] = (float)((double)yr + acc);
}

template <typename V, int SIGMA, bool HUB, int GM>
__global__ void __launch_bounds__(kPersistWarps * 32, 1)
    merbit_persistent_kernel(const MerbitOperand<V, SIGMA> m_in, int tile_num, int nrow, int* __restrict__ ticket,
                             const int32_t* __restrict__ hub_cols, int hub_k, const int32_t* __restrict__ chunk_start,
                             const int4* __restrict__ brun, int* __restrict__ bflag)
{
    extern __shared__ __align__(16) float s_dyn[];
    __shared__ int s_last, s_nlong, s_arrive[2], s_next;
    const int warp = threadIdx.x >> 5;
    const int G = gridDim.x;
    const int chunk = (tile_num + G - 1) / G;
    // chunk c = [start(c), start(c + 1))
    auto start = [&](int c) {
        return chunk_start ? (c >= G ? tile_num : __ldg(chunk_start + c)) : min(c * chunk, tile_num);
    };
    const int t0 = start(blockIdx.x);
    const int t1 = start(blockIdx.x + 1);
    float* s = s_dyn + warp * tile_smem_words<SIGMA>();
    const TilePolicy pol{l2_evict_last_policy(), l2_evict_first_policy()};
    MerbitOperand<V, SIGMA> m = m_in;
    // tiles [t0, t0 + nstat) round robin, the rest from the counter s_next
    const int nstat = (t1 - t0) / kPersistWarps * kStaticNum / kStaticDen * kPersistWarps;
    if (threadIdx.x == 0) s_next = t0 + nstat;
    if constexpr (!HUB) __syncthreads();
    if constexpr (HUB) {
        // stage x of the hub columns once per CTA
        float* hub = s_dyn + kPersistWarps * tile_smem_words<SIGMA>();
        // 16 independent gathers in flight per thread
        constexpr int PF = 16;
        for (int base = threadIdx.x; base < hub_k; base += blockDim.x * PF) {
            int c[PF];
            float v[PF];
#pragma unroll
            for (int j = 0; j < PF; ++j) {
                const int i = base + j * (int)blockDim.x;
                c[j] = i < hub_k ? __ldg(hub_cols + i) : -1;
            }
#pragma unroll
            for (int j = 0; j < PF; ++j) v[j] = c[j] >= 0 ? ld_x(m.x + c[j], pol.x_keep) : 0.f;
#pragma unroll
            for (int j = 0; j < PF; ++j) {
                const int i = base + j * (int)blockDim.x;
                if (i < hub_k) hub[i] = v[j];
            }
        }
        m.hub = hub;
        __syncthreads();
    }
    for (int t = t0 + warp; t < t0 + nstat; t += kPersistWarps) merbit_tile<V, SIGMA, true, HUB, GM>(m, t, s, pol);
    for (;;) {
        int t = 0;
        if ((threadIdx.x & 31) == 0) t = atomicAdd(&s_next, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= t1) break;
        merbit_tile<V, SIGMA, true, HUB, GM>(m, t, s, pol);
    }
    __syncthreads();
    // runs inside the chunk: open rows and carries staged in the (now free)
    // tile staging memory, so a run is walked in shared memory rather than
    // one dependent global load per tile
    constexpr int kStageWords = kPersistWarps * tile_smem_words<SIGMA>();
    const int nt = t1 - t0;
    if (nt <= kStageWords / 2) {
        int* sR = reinterpret_cast<int*>(s_dyn);
        float* sC = s_dyn + kStageWords / 2;
        for (int i = threadIdx.x; i < nt; i += blockDim.x) {
            sR[i] = open_row(m.tile_y, t0 + i);
            sC[i] = m.carry[t0 + i];
        }
        const int r_before = t0 > 0 ? open_row(m.tile_y, t0 - 1) : -1;
        __syncthreads();
        for (int i = threadIdx.x; i < nt; i += blockDim.x) {
            const int R = sR[i];
            if (R >= nrow) continue;
            if (t0 + i > 0 && (i > 0 ? sR[i - 1] : r_before) == R) continue;  // not the first tile of its run
            double acc = 0.0;
            int u = i;
            while (u < nt && sR[u] == R) {
                acc += (double)sC[u];
                ++u;
            }
            if (u >= nt) continue;  // the row ends in a later chunk: boundary pass
            m.y[R] = (float)((double)m.y[R] + acc);
        }
    } else {
        for (int t = t0 + (int)threadIdx.x; t < t1; t += blockDim.x)
            fixup_in_chunk(m.tile_y, m.carry, t0, t1, nrow, m.y, t);
    }
    __threadfence();
    __syncthreads();
    const int lane = threadIdx.x & 31;
    if (brun) {
        // runs that cross a chunk start and lie in the two chunks beside it:
        // the second of the two CTAs to get here finishes the run
        if (threadIdx.x == 0) {
            const int c = blockIdx.x;
            s_arrive[0] = c >= 1 ? atomicAdd(bflag + c, 1) : 0;
            s_arrive[1] = c + 1 <= G - 1 ? atomicAdd(bflag + c + 1, 1) : 0;
            __threadfence();
        }
        __syncthreads();
        if (warp < 2 && s_arrive[warp] == 1) {
            const int c = blockIdx.x + warp;
            const int4 run = __ldg(brun + c);
            if (run.w == 1) finish_run(run, m.carry, m.y, lane);
            if (lane == 0) bflag[c] = 0;  // both have arrived: ready for the next launch
        }
        __threadfence();
        __syncthreads();
    }
    if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1) == G - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (brun) {
        // runs that start before the chunk ahead of their boundary
        int* s_list = reinterpret_cast<int*>(s_dyn);
        if (threadIdx.x == 0) s_nlong = 0;
        __syncthreads();
        for (int c = 1 + (int)threadIdx.x; c < G; c += blockDim.x)
            if (__ldg(&brun[c].w) == 2) s_list[atomicAdd(&s_nlong, 1)] = c;
        __syncthreads();
        for (int i = warp; i < s_nlong; i += kPersistWarps) finish_run(__ldg(brun + s_list[i]), m.carry, m.y, lane);
        if (threadIdx.x == 0) *ticket = 0;  // ready for the next launch
        return;
    }
    // plans without a run table (equal tile counts): the last CTA finishes
    // every crossing run; one thread per boundary finishes a run of one carry
    // tile (the common case: three independent loads, then y); longer runs
    // are listed (in the free staging memory) and finished one warp each
    int* s_long = reinterpret_cast<int*>(s_dyn);
    if (threadIdx.x == 0) s_nlong = 0;
    __syncthreads();
    for (int c = 1 + (int)threadIdx.x; c < G; c += blockDim.x) {
        const int b = start(c);
        if (b <= 0 || b >= tile_num) continue;
        const int R = open_row(m.tile_y, b - 1);
        if (R >= nrow) continue;
        const int r_prev = b >= 2 ? open_row(m.tile_y, b - 2) : -1;
        const int r_next = open_row(m.tile_y, b);
        if (r_prev == R || r_next == R) {
            s_long[atomicAdd(&s_nlong, 1)] = c;
            continue;
        }
        // the run is tile b - 1 alone and its row ends in tile b, finished
        // here when tile b belongs to this chunk (an empty chunk leaves it
        // to the next boundary, which has the same start)
        if (b >= start(c + 1)) continue;
        m.y[R] = (float)((double)__ldcg(m.y + R) + (double)__ldcg(m.carry + b - 1));
    }
    __syncthreads();
    for (int i = warp; i < s_nlong; i += kPersistWarps) {
        const int c = s_long[i];
        fixup_boundary_warp(m.tile_y, m.carry, tile_num, start(c), start(c + 1), nrow, m.y, lane);
    }
    if (threadIdx.x == 0) *ticket = 0;  // ready for the next launch
}

// One thread per tile finishes the short runs that start at its tile; the
// warp then finishes its lanes' long runs together (whole warps: the grid
// covers the tiles in blocks of 256). Launched as a programmatic dependent
// of the SpMV grid: its launch and scheduling overlap that grid's last wave,
// and it waits for that grid's completion (and memory) before any read. In
// an ordinary launch the wait returns at once.
__global__ void merbit_fixup_kernel(const uint32_t* __restrict__ tile_y, const float* __restrict__ carry,
                                    int tile_num, int nrow, float* __restrict__ y)
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int kind = t < tile_num ? fixup_run_short(tile_y, carry, tile_num, nrow, y, t) : 0;
    unsigned long_runs = __ballot_sync(0xffffffffu, kind == 2);
    while (long_runs) {
        const int src = __ffs(long_runs) - 1;
        long_runs &= long_runs - 1;
        fixup_run_warp(tile_y, carry, tile_num, y, __shfl_sync(0xffffffffu, t, src), threadIdx.x & 31);
    }
}

template <typename V, int SIGMA, int WARPS>
static int launch_spmv_t(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x, float* y,
                         float* carry, cudaStream_t st)
{
    const int grid = (p.tile_num + WARPS - 1) / WARPS;
    const int vec_ok = ((reinterpret_cast<uintptr_t>(colidx) & 15) == 0) &&
                       ((reinterpret_cast<uintptr_t>(vals) & (4 * sizeof(V) - 1)) == 0);
    MerbitOperand<V, SIGMA> m;
    m.tile_x = p.tile_x;
    m.tile_y = p.tile_y;
    m.lane_desc = reinterpret_cast<const typename DescOf<SIGMA>::T*>(p.lane_desc);
    m.lane_num = p.lane_num;
    m.nnz = nnz;
    m.items = (int64_t)p.n_rows + p.nnz;
    m.colidx = colidx;
    m.vals = reinterpret_cast<const V*>(vals);
    m.x = x;
    m.y = y;
    m.carry = carry;
    m.vec_ok = vec_ok;
    m.hub = nullptr;
    m.gather_mode = p.gather_mode;
    if (grid > 0) {
        if (p.gather_mode == 0)
            merbit_spmv_kernel<V, SIGMA, WARPS, 0><<<grid, WARPS * 32, 0, st>>>(m, p.tile_num);
        else
            merbit_spmv_kernel<V, SIGMA, WARPS, -1><<<grid, WARPS * 32, 0, st>>>(m, p.tile_num);
    }
    MR_CUDA_TRY(cudaGetLastError());
    if (p.tile_num > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)((p.tile_num + 255) / 256));
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        MR_CUDA_TRY(cudaLaunchKernelEx(&cfg, merbit_fixup_kernel, (const uint32_t*)p.tile_y, (const float*)carry,
                                       p.tile_num, p.n_rows, y));
    }
    return MR_OK;
}

template <typename V, int SIGMA, int GM>
static int launch_persistent(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x,
                             float* y, float* carry, cudaStream_t st)
{
    if (p.tile_num == 0) return MR_OK;
    MerbitOperand<V, SIGMA> m;
    m.tile_x = p.tile_x;
    m.tile_y = p.tile_y;
    m.lane_desc = reinterpret_cast<const typename DescOf<SIGMA>::T*>(p.lane_desc);
    m.lane_num = p.lane_num;
    m.nnz = nnz;
    m.items = (int64_t)p.n_rows + p.nnz;
    const int* cols = p.hub_k > 0 ? p.colh : colidx;  // hub plans read their remapped copy
    m.colidx = cols;
    m.vals = reinterpret_cast<const V*>(vals);
    m.x = x;
    m.y = y;
    m.carry = carry;
    m.vec_ok = ((reinterpret_cast<uintptr_t>(cols) & 15) == 0) &&
               ((reinterpret_cast<uintptr_t>(vals) & (4 * sizeof(V) - 1)) == 0);
    m.hub = nullptr;
    m.gather_mode = p.gather_mode;
    const size_t stage = sizeof(float) * (size_t)kPersistWarps * tile_smem_words<SIGMA>();
    const int grid = persistent_grid(p.tile_num);
    // the plan's bounds were made for this grid (same device model); any
    // other grid takes equal tile counts
    const bool own = p.chunk_start && p.chunks == grid;
    const int32_t* bounds = own ? p.chunk_start : nullptr;
    const int4* brun = own ? p.boundary_run : nullptr;
    int* bflag = own ? p.boundary_flag : nullptr;
    if (p.hub_k > 0) {
        const size_t smem = stage + sizeof(float) * (size_t)p.hub_k;
        static PerDeviceOnce once;
        MR_CUDA_TRY(once.run([&] {
            int optin = 0, dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            cudaFuncAttributes fa;
            cudaError_t e = cudaFuncGetAttributes(&fa, merbit_persistent_kernel<V, SIGMA, true, GM>);
            // static and dynamic shared memory together may not exceed the opt-in limit
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(merbit_persistent_kernel<V, SIGMA, true, GM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         optin - (int)fa.sharedSizeBytes);
            return e;
        }));
        // carve-out sized to this plan's shared memory: the rest stays L1
        const int pct = std::min(100, (int)((smem + 1023) / 1024 * 100 / 228) + 1);
        MR_CUDA_TRY(cudaFuncSetAttribute(merbit_persistent_kernel<V, SIGMA, true, GM>,
                                         cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        merbit_persistent_kernel<V, SIGMA, true, GM><<<grid, kPersistWarps * 32, smem, st>>>(m, p.tile_num, p.n_rows,
                                                                                        p.ticket, p.hub_cols, p.hub_k,
                                                                                        bounds, brun, bflag);
    } else {
        static PerDeviceOnce once;
        MR_CUDA_TRY(once.run([&] {
            cudaError_t e = cudaFuncSetAttribute(merbit_persistent_kernel<V, SIGMA, false, GM>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage);
            // smallest shared-memory carve-out that fits: the rest of the
            // SM's 256 KB stays L1 for x
            const int pct = (int)((stage + 1023) / 1024 * 100 / 228) + 1;
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(merbit_persistent_kernel<V, SIGMA, false, GM>,
                                         cudaFuncAttributePreferredSharedMemoryCarveout, std::min(pct, 100));
            return e;
        }));
        merbit_persistent_kernel<V, SIGMA, false, GM><<<grid, kPersistWarps * 32, stage, st>>>(m, p.tile_num, p.n_rows,
                                                                                          p.ticket, nullptr, 0, bounds,
                                                                                          brun, bflag);
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

// ------------------------------------------------------------ hub cache ----

__global__ void col_count_kernel(const int32_t* __restrict__ colidx, int64_t nnz, int32_t* __restrict__ cnt)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[colidx[k]], 1);
}

constexpr int kCountCap = 1 << 16;

// histogram of column counts (counts >= kCountCap share the last bucket)
__global__ void count_hist_kernel(const int32_t* __restrict__ cnt, int ncols, unsigned long long* __restrict__ h,
                                  unsigned long long* __restrict__ hw)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x) {
        const int v = cnt[c];
        if (v >= 2) {
            atomicAdd(&h[min(v, kCountCap)], 1ull);
            atomicAdd(&hw[min(v, kCountCap)], (unsigned long long)v);
        }
    }
}

__global__ void hub_flag_kernel(const int32_t* __restrict__ cnt, int ncols, int thr, int32_t* __restrict__ flag)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x)
        flag[c] = cnt[c] >= thr ? 1 : 0;
}

// slot = exclusive scan of the flags; hub_cols[slot] = c; slot_of[c] = slot or -1
__global__ void hub_slots_kernel(const int32_t* __restrict__ flag, const int32_t* __restrict__ scan, int ncols,
                                 int32_t* __restrict__ hub_cols, int32_t* __restrict__ slot_of)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x) {
        if (flag[c]) {
            hub_cols[scan[c]] = c;
            slot_of[c] = scan[c];
        } else {
            slot_of[c] = -1;
        }
    }
}

__global__ void hub_remap_kernel(const int32_t* __restrict__ colidx, int64_t nnz, const int32_t* __restrict__ slot_of,
                                 int32_t* __restrict__ colh)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int c = colidx[k];
        const int s = slot_of[c];
        colh[k] = s >= 0 ? (int)(0x80000000u | (uint32_t)s) : c;
    }
}

}  // namespace mr

namespace mr {

int hub_capacity(int sigma)
{
    int optin = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const long long stage = 4ll * kPersistWarps * (32 * sigma + 8);
    // leave 64 KB of the SM's memory as L1. The x gathers that miss the hub
    // hit L1 only ~2% of the time, but every load in flight holds L1 space:
    // on R-MAT s22 (SIGMA 20) a 32 KB reserve costs a third of the
    // throughput although the larger hub serves 50% instead of 44% of the
    // gathers, and a smaller hub (more L1) is slower again (-1% at 16K
    // columns, -7% at 4K)
    const long long room = (long long)optin - stage - 65536 - 1024;
    if (room <= 0) return 0;
    return (int)std::min<long long>(room / 4 / 128 * 128, 1 << 20);
}

int build_hub_cache(MerbitPlan& p, const mr_csr_view& A, cudaStream_t st)
{
    p.hub_k = 0;
    p.hub_coverage = 0.0;
    int cap = hub_capacity(p.sigma);
    if (p.hub_limit > 0) cap = std::min(cap, p.hub_limit);
    if (cap < 1024 || A.nnz < (1 << 16) || A.n_cols <= 0) return MR_OK;
    const int ncols = A.n_cols;
    const int grid_c = (int)std::min<int64_t>(((int64_t)ncols + 255) / 256, (int64_t)sm_count() * 8);
    const int grid_k = (int)std::min<int64_t>((A.nnz + 255) / 256, (int64_t)sm_count() * 16);
    DevBuf cnt, hist, flag, scan, slot_of;
    MR_TRY(cnt.alloc(sizeof(int32_t) * (size_t)ncols, st));
    MR_TRY(hist.alloc(sizeof(unsigned long long) * 2 * (kCountCap + 1), st));
    MR_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (size_t)ncols, st));
    MR_CUDA_TRY(cudaMemsetAsync(hist.p, 0, sizeof(unsigned long long) * 2 * (kCountCap + 1), st));
    col_count_kernel<<<grid_k, 256, 0, st>>>(A.colidx, A.nnz, cnt.as<int32_t>());
    unsigned long long* h = hist.as<unsigned long long>();
    count_hist_kernel<<<grid_c, 256, 0, st>>>(cnt.as<int32_t>(), ncols, h, h + kCountCap + 1);
    MR_CUDA_TRY(cudaGetLastError());
    std::vector<unsigned long long> hh(2 * (kCountCap + 1));
    MR_CUDA_TRY(cudaMemcpyAsync(hh.data(), h, sizeof(unsigned long long) * hh.size(), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    // smallest threshold thr >= 2 whose column set {count >= thr} fits
    unsigned long long ncol = 0, weight = 0;
    int thr = kCountCap + 1;
    for (int c = kCountCap; c >= 2; --c) {
        if (ncol + hh[(size_t)c] > (unsigned long long)cap) break;
        ncol += hh[(size_t)c];
        weight += hh[(size_t)(kCountCap + 1 + c)];
        thr = c;
    }
    const double coverage = (double)weight / (double)A.nnz;
    // a hub cache that serves few gathers is not worth its shared memory
    // (the L1 it displaces would serve them as well): below 20% of the
    // nonzeros the plan runs without it
    if (ncol == 0 || coverage < 0.20) return MR_OK;
    MR_TRY(flag.alloc(sizeof(int32_t) * (size_t)ncols, st));
    MR_TRY(scan.alloc(sizeof(int32_t) * ((size_t)ncols + 1), st));
    MR_TRY(slot_of.alloc(sizeof(int32_t) * (size_t)ncols, st));
    hub_flag_kernel<<<grid_c, 256, 0, st>>>(cnt.as<int32_t>(), ncols, thr, flag.as<int32_t>());
    MR_TRY(exclusive_scan_i32(flag.as<int32_t>(), scan.as<int32_t>(), ncols, st));
    if (cudaMalloc(&p.hub_cols, sizeof(int32_t) * (size_t)ncol) != cudaSuccess ||
        cudaMalloc(&p.colh, sizeof(int32_t) * (size_t)A.nnz) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p.hub_cols);
        cudaFree(p.colh);
        p.hub_cols = nullptr;
        p.colh = nullptr;
        return MR_OK;  // no room for the cache: run without it
    }
    hub_slots_kernel<<<grid_c, 256, 0, st>>>(flag.as<int32_t>(), scan.as<int32_t>(), ncols, p.hub_cols,
                                            slot_of.as<int32_t>());
    hub_remap_kernel<<<grid_k, 256, 0, st>>>(A.colidx, A.nnz, slot_of.as<int32_t>(), p.colh);
    MR_CUDA_TRY(cudaGetLastError());
    p.hub_k = (int)ncol;
    p.hub_coverage = coverage;
    return MR_OK;
}

void free_plan_buffers(MerbitPlan& p)
{
    cudaFree(p.tile_x);
    cudaFree(p.tile_y);
    cudaFree(p.lane_desc);
    cudaFree(p.carry);
    cudaFree(p.ticket);
    cudaFree(p.colh);
    cudaFree(p.hub_cols);
    cudaFree(p.chunk_start);
    cudaFree(p.boundary_run);
    cudaFree(p.boundary_flag);
}

int persistent_grid(int tile_num)
{
    return std::max(1, std::min(sm_count(), (tile_num + kPersistWarps - 1) / kPersistWarps));
}

// Estimated cost of each tile, one warp per tile: 8 per x gather that misses
// the hub cache (an L2 access), 1 per nonzero (stream bytes and hub gathers)
// and 8 per tile. On R-MAT s21 under equal tile counts the SMs' busy cycles
// spread as their chunks' non-hub gathers do (max / mean 1.21 measured, 1.19
// predicted); weights of 4 to 32 per miss time the same at s22.
constexpr int kCostMiss = 8;
constexpr int kCostTile = 8;

__global__ void tile_cost_kernel(const uint32_t* __restrict__ tile_x, const int32_t* __restrict__ cols, int nnz,
                                 int tile_num, int32_t* __restrict__ cost)
{
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ws = (gridDim.x * blockDim.x) >> 5;
    for (int t = w; t < tile_num; t += ws) {
        const int a = min((int)__ldg(tile_x + t), nnz);
        const int b = min((int)__ldg(tile_x + t + 1), nnz);
        int miss = 0;
        for (int k = a + lane; k < b; k += 32) miss += __ldg(cols + k) >= 0 ? 1 : 0;
        miss = __reduce_add_sync(0xffffffffu, miss);
        if (lane == 0) cost[t] = kCostMiss * miss + (b - a) + kCostTile;
    }
}

int build_chunk_bounds(MerbitPlan& p, const int* colidx, cudaStream_t st)
{
    const int G = persistent_grid(p.tile_num);
    if (G < 2 || p.tile_num < 2 * G) return MR_OK;  // equal tile counts
    const int* cols = p.hub_k > 0 ? p.colh : colidx;
    DevBuf cost;
    MR_TRY(cost.alloc(sizeof(int32_t) * (size_t)p.tile_num, st));
    const int grid = (int)std::min<int64_t>(((int64_t)p.tile_num * 32 + 255) / 256, (int64_t)sm_count() * 16);
    tile_cost_kernel<<<grid, 256, 0, st>>>(p.tile_x, cols, (int)p.nnz, p.tile_num, cost.as<int32_t>());
    MR_CUDA_TRY(cudaGetLastError());
    std::vector<int32_t> c((size_t)p.tile_num);
    MR_CUDA_TRY(cudaMemcpyAsync(c.data(), cost.p, sizeof(int32_t) * c.size(), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    // chunk g starts at the first tile whose cost prefix reaches g / G of the total
    std::vector<int64_t> pre((size_t)p.tile_num + 1, 0);
    for (int t = 0; t < p.tile_num; ++t) pre[(size_t)t + 1] = pre[(size_t)t] + c[(size_t)t];
    const int64_t total = pre.back();
    std::vector<int32_t> bounds((size_t)G + 1);
    for (int g = 0; g <= G; ++g) {
        const int64_t target = (int64_t)((__int128)total * g / G);
        bounds[(size_t)g] = (int32_t)(std::lower_bound(pre.begin(), pre.end(), target) - pre.begin());
    }
    bounds[0] = 0;
    bounds[(size_t)G] = p.tile_num;
    // the carry run crossing each chunk start (the same runs, found the same
    // way, as the kernel's boundary pass over tile_y)
    std::vector<uint32_t> ty((size_t)p.tile_num + 1);
    MR_CUDA_TRY(cudaMemcpy(ty.data(), p.tile_y, sizeof(uint32_t) * ty.size(), cudaMemcpyDeviceToHost));
    auto orow = [&](int t) { return (int)(ty[(size_t)t + 1] & 0x7fffffffu); };
    std::vector<int4> runs((size_t)G + 1, int4{0, 0, 0, 0});
    for (int c = 1; c < G; ++c) {
        const int a = bounds[(size_t)c - 1], b = bounds[(size_t)c], e = bounds[(size_t)c + 1];
        if (b <= 0 || b >= p.tile_num || b >= e) continue;
        const int R = orow(b - 1);
        if (R >= p.n_rows) continue;
        int ue = b - 1;
        while (ue + 1 < p.tile_num && orow(ue + 1) == R) ++ue;
        if (ue + 1 >= e) continue;  // the row ends in a later chunk
        int u0 = b - 1;
        while (u0 > 0 && orow(u0 - 1) == R) --u0;
        runs[(size_t)c] = int4{R, u0, ue, (a < b && u0 >= a) ? 1 : 2};
    }
    auto release = [&] {
        cudaFree(p.chunk_start);
        cudaFree(p.boundary_run);
        cudaFree(p.boundary_flag);
        p.chunk_start = nullptr;
        p.boundary_run = nullptr;
        p.boundary_flag = nullptr;
    };
    if (cudaMalloc(&p.chunk_start, sizeof(int32_t) * bounds.size()) != cudaSuccess ||
        cudaMalloc(&p.boundary_run, sizeof(int4) * runs.size()) != cudaSuccess ||
        cudaMalloc(&p.boundary_flag, sizeof(int) * runs.size()) != cudaSuccess) {
        cudaGetLastError();
        release();
        return MR_OK;  // no room: equal tile counts
    }
    if (cudaMemcpyAsync(p.chunk_start, bounds.data(), sizeof(int32_t) * bounds.size(), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(p.boundary_run, runs.data(), sizeof(int4) * runs.size(), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemsetAsync(p.boundary_flag, 0, sizeof(int) * runs.size(), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {  // the host vectors go out of scope
        release();
        return MR_ERR_CUDA;
    }
    p.chunks = G;
    return MR_OK;
}

}  // namespace mr

namespace mr {

template <typename V, int SIGMA>
static int launch_spmv_w(const MerbitPlan& p, const int* colidx, const void* vals, int nnz, const float* x, float* y,
                         float* carry, cudaStream_t st)
{
    switch (p.block) {
    case 1024:
        return p.gather_mode == 0 ? launch_persistent<V, SIGMA, 0>(p, colidx, vals, nnz, x, y, carry, st)
                                  : launch_persistent<V, SIGMA, -1>(p, colidx, vals, nnz, x, y, carry, st);
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
