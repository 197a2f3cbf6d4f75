// One MERBIT tile (32 lanes x SIGMA merge items) processed by one warp.
// Shared by the single-matrix kernel (merbit.cu) and the batched persistent
// kernel (batch.cu).
//
// Plan format (the reference's, include/merbit.cuh:84-131): lane descriptor
// = flags << (18|22) | delta_row << (9|11) | delta_nz; tile_x = first nonzero
// of the tile, tile_y = first row, bit 31 = all items are nonzeros of one row.
//
// Per tile: (1) every independent load is issued up front (tile bounds, the
// lane's descriptor); (2) colidx/values of the tile are streamed as 16-byte
// evict-first vectors, all vector loads of a round before any dependent x
// gather, x gathered with an L2 evict-last policy, products staged in shared
// memory; (3) each lane walks its SIGMA items from its descriptor, finished
// rows stay in registers; (4) a warp segmented scan carries the partial sum
// of a row across lanes; (5) finished rows leave through shared memory as
// coalesced streaming stores, and the sum still open at the tile end goes to
// carry[tile] for the FP64 fix-up. No atomics anywhere.
#ifndef MR_MERBIT_TILE_CUH
#define MR_MERBIT_TILE_CUH

#include <type_traits>

#include "common.cuh"

namespace mr {

template <int SIGMA> struct DescOf {
    using T = typename std::conditional<(SIGMA < 15), uint32_t, unsigned long long>::type;
    static constexpr int sh_flag = SIGMA < 15 ? 18 : 22;
    static constexpr int sh_dy = SIGMA < 15 ? 9 : 11;
    static constexpr unsigned mask_d = SIGMA < 15 ? 0x1ffu : 0x7ffu;
};

// Shared-memory words per warp: products of one tile (<= 32*SIGMA), shifted
// by up to 3 so that 16-byte vectors stay aligned, plus slack.
template <int SIGMA> constexpr int tile_smem_words() { return 32 * SIGMA + 8; }

template <typename V, int SIGMA> struct MerbitOperand {
    const uint32_t* tile_x;
    const uint32_t* tile_y;
    const typename DescOf<SIGMA>::T* lane_desc;
    int lane_num;
    int nnz;
    int64_t items;  // n_rows + nnz
    const int* colidx;
    const V* vals;
    const float* x;
    float* y;
    float* carry;
    int vec_ok;     // colidx/vals aligned for vector loads
    const float* hub;  // shared-memory x values of hub columns, or nullptr
    int gather_mode;   // ld_x_mode variant of the x gathers
};

// Cache policies of one tile: x gathers keep their lines in L2 (evict-last);
// with NA the matrix streams bypass L1 and are evict-first in L2, so that
// L1 caches only x.
struct TilePolicy {
    uint64_t x_keep;
    uint64_t stream_first;
};

template <bool NA, typename T> __device__ __forceinline__ T ld_s(const T* p, uint64_t pol)
{
    if constexpr (NA)
        return ld_na(p, pol);
    else
        return ld_stream(p);
}

// x[c] for one nonzero. Hub plans mark columns staged in shared memory by the
// sign bit (slot in the low bits). GM = 0 is the default gather (read-only
// path, L2 evict-last) fixed at compile time, so the hot path has no mode
// test per gather; GM = -1 reads m.gather_mode (the plan's tuning flags).
template <bool HUB, int GM, typename V, int SIGMA>
__device__ __forceinline__ float gather_x(const MerbitOperand<V, SIGMA>& m, int c, uint64_t pol)
{
    if constexpr (HUB)
        if (c < 0) return m.hub[c & 0x7fffffff];
    if constexpr (GM == 0)
        return ld_x(m.x + c, pol);
    else
        return ld_x_mode(m.x + c, pol, m.gather_mode);
}

template <typename V, int SIGMA, bool NA = false, bool HUB = false, int GM = 0>
__device__ __forceinline__ void merbit_tile(const MerbitOperand<V, SIGMA>& m, const int tile, float* __restrict__ s,
                                            const TilePolicy pols)
{
    const uint64_t pol = pols.x_keep;
    using D = DescOf<SIGMA>;
    using DT = typename D::T;
    const int lid = threadIdx.x & 31;
    const int gid = tile * 32 + lid;

    // ---- independent loads first ------------------------------------------
    const int x0 = (int)__ldg(m.tile_x + tile);
    const int x1 = (int)__ldg(m.tile_x + tile + 1);
    const uint32_t ty0 = __ldg(m.tile_y + tile);
    const int y1 = (int)(__ldg(m.tile_y + tile + 1) & 0x7fffffffu);
    DT d = 0;
    if (gid < m.lane_num) d = ld_s<NA>(m.lane_desc + gid, pols.stream_first);
    const int y0 = (int)(ty0 & 0x7fffffffu);
    const bool single_row = (ty0 >> 31) != 0;

    // ---- stage products vals[k] * x[colidx[k]] for k in [x0, x1) ---------
    constexpr int NV = 8 * SIGMA + 1;  // max 4-element vectors per tile
    constexpr int ITERS = (NV + 31) / 32;
    constexpr int UNR = ITERS < 4 ? ITERS : 4;
    const int a0 = x0 & ~3;  // 16-byte aligned start (FP32 / int32)
    const int shift = x0 - a0;
    const int nvec = (x1 - a0 + 3) >> 2;
    float part = 0.f;
#pragma unroll 1
    for (int base = 0; base < ITERS; base += UNR) {
        int col[UNR][4];
        float val[UNR][4];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int v = lid + 32 * (base + u);
            const int k = a0 + 4 * v;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                col[u][j] = 0;
                val[u][j] = 0.f;
            }
            if (v < nvec) {
                if (m.vec_ok && k + 3 < m.nnz) {
                    const int4 c = ld_s<NA>(reinterpret_cast<const int4*>(m.colidx + k), pols.stream_first);
                    col[u][0] = c.x;
                    col[u][1] = c.y;
                    col[u][2] = c.z;
                    col[u][3] = c.w;
                    Vec4<V>::unpack(ld_s<NA>(reinterpret_cast<const typename Vec4<V>::T*>(m.vals + k), pols.stream_first),
                                    val[u]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int kk = k + j;
                        if (kk >= x0 && kk < x1) {
                            col[u][j] = ld_stream(m.colidx + kk);
                            val[u][j] = ValueTraits<V>::f(ld_stream(m.vals + kk));
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int v = lid + 32 * (base + u);
            if (v < nvec) {
                const int k = a0 + 4 * v;
                float p[4];
                if (!single_row) {
                    // products outside [x0, x1) land in staging slots that
                    // the walk never reads: no per-element range test. Their
                    // column indices are real entries of neighbouring tiles
                    // (vector path) or 0 (edge path), so every gather is in
                    // bounds.
#pragma unroll
                    for (int j = 0; j < 4; ++j) p[j] = val[u][j] * gather_x<HUB, GM>(m, col[u][j], pol);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        p[j] = (k + j >= x0 && k + j < x1) ? val[u][j] * gather_x<HUB, GM>(m, col[u][j], pol) : 0.f;
                }
                if (single_row)
                    part += (p[0] + p[1]) + (p[2] + p[3]);
                else
                    *reinterpret_cast<float4*>(s + 4 * v) = make_float4(p[0], p[1], p[2], p[3]);
            }
        }
    }
    if (single_row) {
        // every item of this tile is a nonzero of row y0 (== y1): the whole
        // tile is a carry into that row
        part = warp_sum(part);
        if (lid == 0) m.carry[tile] = part;
        return;
    }
    __syncwarp();

    // ---- walk this lane's SIGMA merge items -------------------------------
    const int lane_items = gid < m.lane_num ? (int)min64((int64_t)SIGMA, m.items - (int64_t)gid * SIGMA) : 0;
    const uint32_t flags =
        (uint32_t)(d >> D::sh_flag) & ((lane_items >= 32) ? 0xffffffffu : ((1u << lane_items) - 1u));
    int xi = shift + (int)(d & D::mask_d);
    const int dy = (int)((d >> D::sh_dy) & D::mask_d);

    float rows[SIGMA];  // finished row sums, indexed by the item that ends them
    float cur = 0.f;
    // every lane of a tile before the last holds SIGMA items: that walk
    // needs no per-item range test
    if ((int64_t)(tile + 1) * 32 * SIGMA <= m.items) {
#pragma unroll
        for (int i = 0; i < SIGMA; ++i) {
            rows[i] = 0.f;
            if ((flags >> i) & 1u) {
                rows[i] = cur;
                cur = 0.f;
            } else {
                cur += s[xi];
                ++xi;
            }
        }
    } else {
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
    }
    const int first = flags ? (__ffs(flags) - 1) : SIGMA;
    float head = 0.f;
#pragma unroll
    for (int i = 0; i < SIGMA; ++i)
        if (i == first) head = rows[i];

    // ---- warp segmented scan of the carried partial sums ------------------
    // a lane passes on its sum after its last row end; a lane with a row end
    // starts a new segment
    float incl = cur;
    bool seg = flags != 0;
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
    for (int j = lid; j < nrows; j += 32) __stcs(m.y + y0 + j, s[j]);
    if (lid == 0) m.carry[tile] = tile_carry;
    __syncwarp();  // the warp may reuse s for its next tile
}

// Carry runs. A run is the tiles t, t+1, ... whose row still open at the
// tile end is the same row R (tile_y[u + 1] == R); their carries are added
// to y[R] in FP64 in tile order, once the tile where R ends has written it.
__device__ __forceinline__ int tile_open_row(const uint32_t* __restrict__ tile_y, int t)
{
    return (int)(__ldg(tile_y + t + 1) & 0x7fffffffu);
}

constexpr int kShortRun = 8;

// For tile t: 0 if it does not start a run; 1 if it starts a run of at most
// kShortRun tiles, now finished (the open rows and carries of the next tiles
// are loaded together, then summed in order); 2 if it starts a longer run,
// left to fixup_run_warp.
__device__ __forceinline__ int fixup_run_short(const uint32_t* __restrict__ tile_y, const float* __restrict__ carry,
                                               int tile_num, int nrow, float* __restrict__ y, int t)
{
    const int R = tile_open_row(tile_y, t);
    if (R >= nrow) return 0;
    if (t > 0 && tile_open_row(tile_y, t - 1) == R) return 0;  // not the first tile of its run
    int len = 1;
#pragma unroll
    for (int j = 1; j <= kShortRun; ++j) {
        const bool same = t + j < tile_num && tile_open_row(tile_y, t + j) == R;
        if (same && len == j) len = j + 1;
    }
    if (len > kShortRun) return 2;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kShortRun; ++j)
        if (j < len) acc += (double)__ldg(carry + t + j);
    y[R] = (float)((double)y[R] + acc);
    return 1;
}

// The run starting at tile t, by the whole warp: its end found 32 tiles per
// step with ballots (open rows never decrease along the tiles), its carries
// loaded 32 at a time and summed in FP64 in tile order through shuffles.
__device__ __forceinline__ void fixup_run_warp(const uint32_t* __restrict__ tile_y, const float* __restrict__ carry,
                                               int tile_num, float* __restrict__ y, int t, int lane)
{
    const int R = tile_open_row(tile_y, t);
    int ue = t;
    for (;;) {
        const int q = ue + 1 + lane;
        const unsigned m = __ballot_sync(0xffffffffu, q < tile_num && tile_open_row(tile_y, q) == R);
        if (m != 0xffffffffu) {
            ue += __ffs(~m) - 1;
            break;
        }
        ue += 32;
    }
    double acc = 0.0;
    for (int base = t; base <= ue; base += 32) {
        const float c = base + lane <= ue ? __ldg(carry + base + lane) : 0.f;
        const int cnt = min(32, ue - base + 1);
        for (int j = 0; j < cnt; ++j) acc += (double)__shfl_sync(0xffffffffu, c, j);
    }
    if (lane == 0) y[R] = (float)((double)y[R] + acc);
}

}  // namespace mr

#endif
