// Batched MERBIT SpMV: many independent matrices in one persistent launch,
// replayable as a CUDA graph, plus the (SIGMA, BLOCK) autotuner.
//
// Items are grouped by (SIGMA, value dtype). Each group keeps in device
// memory a table of per-item operands and the exclusive prefix of their tile
// counts; one persistent kernel per group walks the concatenated tile space
// (warp w takes tiles w, w + W, ... over the whole grid), finds each tile's
// item by binary search in the prefix and runs the same tile routine as the
// single-matrix kernel; one fix-up kernel per group finishes the rows that
// span tiles. Every item has its own carry scratch, so one plan may appear in
// several items, and each item's result is bitwise the same as a
// single-matrix mr_spmv_merbit of it (same tiles, same order of operations).
// Changing an item's x/y pointers rewrites the device table only, so a
// captured graph stays valid.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <cmath>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "internal.hpp"
#include "merbit_tile.cuh"

using namespace mr;

namespace mr {

template <typename V, int SIGMA> struct BatchOp {
    MerbitOperand<V, SIGMA> m;
    int tile_num;
    int n_rows;
};

// item owning global tile g: largest i with prefix[i] <= g
__device__ __forceinline__ int find_item(const long long* __restrict__ prefix, int count, long long g)
{
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One 1024-thread CTA per SM over the concatenated tile space of the group's
// items, in 32-tile sub-chunks (one tile per warp), so the warps of an SM
// work on neighbouring tiles of the same item (x reuse in L1, the streams
// bypass L1 and leave L2 first). A warp looks its item up again only when
// its tile leaves the current item.
constexpr int kBatchWarps = 32;

template <typename V, int SIGMA>
__global__ void __launch_bounds__(kBatchWarps * 32, 1)
    batch_spmv_kernel(const BatchOp<V, SIGMA>* __restrict__ ops, const long long* __restrict__ prefix, int count,
                      long long total_tiles)
{
    extern __shared__ __align__(16) float s_dyn[];
    const int warp = threadIdx.x >> 5;
    float* s = s_dyn + warp * tile_smem_words<SIGMA>();
    const TilePolicy pol{l2_evict_last_policy(), l2_evict_first_policy()};
    // CTAs take 32-tile sub-chunks round-robin (CTA b: sub-chunks b, b + G,
    // ...), so every CTA samples the whole group: items whose tiles cost
    // different amounts (banded rows gather from L1, power-law rows from L2)
    // average out, where contiguous chunks left the slowest SM 26% above the
    // mean. Warp w of the CTA takes tile w of the sub-chunk, so the 32 warps
    // still work on 32 adjacent tiles. The fix-up is a separate pass over
    // all tiles, so which CTA sums a tile does not matter.
    const long long nsub = (total_tiles + kBatchWarps - 1) / kBatchWarps;
    int it = 0;
    long long lo = 0, hi = 0;
    for (long long sc = blockIdx.x; sc < nsub; sc += gridDim.x) {
        const long long g = sc * kBatchWarps + warp;
        if (g >= total_tiles) continue;
        if (g < lo || g >= hi) {
            it = find_item(prefix, count, g);
            lo = __ldg(prefix + it);
            hi = __ldg(prefix + it + 1);
        }
        // fields read where used (registers are scarce; staging the operand in
        // shared memory measured the same)
        const MerbitOperand<V, SIGMA>& m = ops[it].m;
        const int tile = (int)(g - lo);
        if (m.gather_mode == 0)  // warp-uniform: the default gather without a per-gather mode test
            merbit_tile<V, SIGMA, true, false, 0>(m, tile, s, pol);
        else
            merbit_tile<V, SIGMA, true, false, -1>(m, tile, s, pol);
    }
}

template <typename V, int SIGMA>
__global__ void batch_fixup_kernel(const BatchOp<V, SIGMA>* __restrict__ ops, const long long* __restrict__ prefix,
                                   int count, long long total_tiles)
{
    // warps step over the tiles 32 at a time (the loop is warp-uniform): a
    // lane finishes the short run starting at its tile, then the warp
    // finishes its lanes' long runs together
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = ((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5) * 32; base < total_tiles;
         base += warps * 32) {
        const long long g = base + lane;
        int it = 0, t = 0, kind = 0;
        if (g < total_tiles) {
            it = find_item(prefix, count, g);
            t = (int)(g - __ldg(prefix + it));
            const BatchOp<V, SIGMA>& op = ops[it];
            kind = fixup_run_short(op.m.tile_y, op.m.carry, op.tile_num, op.n_rows, op.m.y, t);
        }
        unsigned long_runs = __ballot_sync(0xffffffffu, kind == 2);
        while (long_runs) {
            const int src = __ffs(long_runs) - 1;
            long_runs &= long_runs - 1;
            const BatchOp<V, SIGMA>& op = ops[__shfl_sync(0xffffffffu, it, src)];
            fixup_run_warp(op.m.tile_y, op.m.carry, op.tile_num, op.m.y, __shfl_sync(0xffffffffu, t, src), lane);
        }
    }
}

}  // namespace mr

// ------------------------------------------------------------------ host ---


namespace {


struct Group {
    int sigma = 14;
    int dtype = MR_F32;
    std::vector<int> items;          // indices into the batch's item list
    void* ops = nullptr;             // device BatchOp<V,SIGMA>[count]
    size_t op_bytes = 0;             // sizeof(BatchOp<V,SIGMA>)
    std::vector<unsigned char> host_ops;
    long long* prefix = nullptr;     // device [count + 1]
    long long total_tiles = 0;
    int grid = 0;
};

template <typename V, int SIGMA> size_t op_size() { return sizeof(BatchOp<V, SIGMA>); }

template <typename V, int SIGMA>
void fill_op(unsigned char* dst, const MerbitPlan& p, const mr_csr_view& A, const float* x, float* y, float* carry)
{
    BatchOp<V, SIGMA> op;
    op.m.tile_x = p.tile_x;
    op.m.tile_y = p.tile_y;
    op.m.lane_desc = reinterpret_cast<const typename DescOf<SIGMA>::T*>(p.lane_desc);
    op.m.lane_num = p.lane_num;
    op.m.nnz = (int)p.nnz;
    op.m.items = (int64_t)p.n_rows + p.nnz;
    op.m.colidx = A.colidx;
    op.m.vals = reinterpret_cast<const V*>(A.vals);
    op.m.x = x;
    op.m.y = y;
    op.m.carry = carry;
    op.m.hub = nullptr;
    op.m.gather_mode = p.gather_mode;
    op.m.vec_ok = ((reinterpret_cast<uintptr_t>(A.colidx) & 15) == 0) &&
                  ((reinterpret_cast<uintptr_t>(A.vals) & (4 * sizeof(V) - 1)) == 0);
    op.tile_num = p.tile_num;
    op.n_rows = p.n_rows;
    std::memcpy(dst, &op, sizeof op);
}

template <typename V, int SIGMA>
int launch_group_t(const Group& g, cudaStream_t st)
{
    if (g.total_tiles == 0) return MR_OK;
    const auto* ops = reinterpret_cast<const BatchOp<V, SIGMA>*>(g.ops);
    const size_t smem = sizeof(float) * (size_t)kBatchWarps * tile_smem_words<SIGMA>();
    static PerDeviceOnce once;
    MR_CUDA_TRY(once.run([&] {
        cudaError_t e =
            cudaFuncSetAttribute(batch_spmv_kernel<V, SIGMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        // smallest shared-memory carve-out that fits: the rest stays L1 for x
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(batch_spmv_kernel<V, SIGMA>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     std::min(100, (int)((smem + 1023) / 1024 * 100 / 228) + 1));
        return e;
    }));
    batch_spmv_kernel<V, SIGMA><<<g.grid, kBatchWarps * 32, smem, st>>>(ops, g.prefix, (int)g.items.size(),
                                                                       g.total_tiles);
    MR_CUDA_TRY(cudaGetLastError());
    const int fg = (int)std::max<long long>(1, std::min<long long>((g.total_tiles + 255) / 256, sm_count() * 8));
    batch_fixup_kernel<V, SIGMA><<<fg, 256, 0, st>>>(ops, g.prefix, (int)g.items.size(), g.total_tiles);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

// dispatch on (dtype, sigma): F is called as F.template operator()<V, SIGMA>()
template <typename F> int dispatch(int dtype, int sigma, F&& f)
{
#define MR_BSIG(V, S) \
    case S: return f.template run<V, S>();
#define MR_BSIGS(V)                                                                                         \
    switch (sigma) {                                                                                        \
        MR_BSIG(V, 7) MR_BSIG(V, 10) MR_BSIG(V, 14) MR_BSIG(V, 16) MR_BSIG(V, 20) MR_BSIG(V, 24) MR_BSIG(V, 28) \
        MR_BSIG(V, 32)                                                                                      \
    default: return MR_ERR_UNSUPPORTED;                                                                     \
    }
    switch (dtype) {
    case MR_F32: MR_BSIGS(float)
    case MR_F16: MR_BSIGS(__half)
    case MR_BF16: MR_BSIGS(__nv_bfloat16)
    default: return MR_ERR_UNSUPPORTED;
    }
#undef MR_BSIGS
#undef MR_BSIG
}

struct OpSizeF {
    template <typename V, int S> int run() { return (int)op_size<V, S>(); }
};
struct LaunchF {
    const Group* g;
    cudaStream_t st;
    template <typename V, int S> int run() { return launch_group_t<V, S>(*g, st); }
};
struct FillF {
    unsigned char* dst;
    const MerbitPlan* p;
    const mr_csr_view* A;
    const float* x;
    float* y;
    float* carry;
    template <typename V, int S> int run()
    {
        fill_op<V, S>(dst, *p, *A, x, y, carry);
        return MR_OK;
    }
};

}  // namespace

namespace mr {

// internal entry points for other host components (the serving loop)
size_t batch_op_bytes(int dtype, int sigma) { return (size_t)dispatch(dtype, sigma, OpSizeF{}); }

int batch_fill_op(void* dst, int dtype, int sigma, const MerbitPlan& p, const mr_csr_view& A, const float* x, float* y,
                  float* carry)
{
    FillF f{static_cast<unsigned char*>(dst), &p, &A, x, y, carry};
    return dispatch(dtype, sigma, f);
}

int batch_launch_ops(int dtype, int sigma, const void* d_ops, const long long* d_prefix, int count,
                     long long total_tiles, cudaStream_t st)
{
    Group g;
    g.dtype = dtype;
    g.sigma = sigma;
    g.items.resize((size_t)count);
    g.ops = const_cast<void*>(d_ops);
    g.prefix = const_cast<long long*>(d_prefix);
    g.total_tiles = total_tiles;
    g.grid = (int)std::max<long long>(
        1, std::min<long long>((total_tiles + kBatchWarps - 1) / kBatchWarps, (long long)sm_count()));
    const int rc = dispatch(dtype, sigma, LaunchF{&g, st});
    g.ops = nullptr;
    g.prefix = nullptr;
    return rc;
}

}  // namespace mr

struct mr_batch {
    std::vector<mr_batch_item> items;
    std::vector<Group> groups;
    std::vector<int> item_group, item_slot;
    std::vector<long long> carry_off;
    float* carry = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
};

static void free_batch(mr_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto& g : b->groups) {
        cudaFree(g.ops);
        cudaFree(g.prefix);
    }
    cudaFree(b->carry);
}

extern "C" {

int mr_batch_create(const mr_batch_item* items, int32_t count, void* stream, mr_batch** out)
{
    if (!out || count < 0 || (count > 0 && !items)) return MR_ERR_INVALID_ARG;
    *out = nullptr;
    cudaStream_t st = as_stream(stream);
    auto* b = new (std::nothrow) mr_batch;
    if (!b) return MR_ERR_NOMEM;
    cudaGetDevice(&b->device);
    b->items.assign(items, items + count);
    b->item_group.resize((size_t)count);
    b->item_slot.resize((size_t)count);
    b->carry_off.resize((size_t)count);
    long long carry_total = 0;
    std::map<std::pair<int, int>, int> gid;
    for (int i = 0; i < count; ++i) {
        const mr_batch_item& it = items[i];
        if (!it.plan) {
            delete b;
            return MR_ERR_INVALID_ARG;
        }
        const MerbitPlan& p = it.plan->p;
        if (it.A.n_rows != p.n_rows || it.A.nnz != p.nnz || !merbit_sigma_supported(p.sigma) ||
            (p.n_rows > 0 && (!it.y || (p.nnz > 0 && (!it.x || !it.A.colidx || !it.A.vals))))) {
            delete b;
            return MR_ERR_INVALID_ARG;
        }
        auto key = std::make_pair(p.sigma, (int)it.A.dtype);
        auto f = gid.find(key);
        int g;
        if (f == gid.end()) {
            g = (int)b->groups.size();
            gid[key] = g;
            b->groups.emplace_back();
            b->groups.back().sigma = p.sigma;
            b->groups.back().dtype = it.A.dtype;
        } else {
            g = f->second;
        }
        b->item_group[(size_t)i] = g;
        b->item_slot[(size_t)i] = (int)b->groups[(size_t)g].items.size();
        b->groups[(size_t)g].items.push_back(i);
        b->carry_off[(size_t)i] = carry_total;
        carry_total += std::max(p.tile_num, 1);
    }
    if (cudaMalloc(&b->carry, sizeof(float) * (size_t)std::max<long long>(carry_total, 1)) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return MR_ERR_NOMEM;
    }
    for (auto& g : b->groups) {
        const int n = (int)g.items.size();
        g.op_bytes = (size_t)dispatch(g.dtype, g.sigma, OpSizeF{});
        g.host_ops.assign(g.op_bytes * n, 0);
        std::vector<long long> prefix((size_t)n + 1, 0);
        for (int k = 0; k < n; ++k) {
            const int i = g.items[(size_t)k];
            const mr_batch_item& it = b->items[(size_t)i];
            FillF f{g.host_ops.data() + g.op_bytes * k, &it.plan->p, &it.A, it.x, it.y, b->carry + b->carry_off[(size_t)i]};
            dispatch(g.dtype, g.sigma, f);
            prefix[(size_t)k + 1] = prefix[(size_t)k] + it.plan->p.tile_num;
        }
        g.total_tiles = prefix[(size_t)n];
        g.grid = (int)std::max<long long>(
            1, std::min<long long>((g.total_tiles + kBatchWarps - 1) / kBatchWarps, (long long)sm_count()));
        if (cudaMalloc(&g.ops, std::max<size_t>(g.host_ops.size(), 16)) != cudaSuccess ||
            cudaMalloc(&g.prefix, sizeof(long long) * prefix.size()) != cudaSuccess) {
            cudaGetLastError();
            free_batch(b);
            delete b;
            return MR_ERR_NOMEM;
        }
        cudaMemcpyAsync(g.ops, g.host_ops.data(), g.host_ops.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g.prefix, prefix.data(), sizeof(long long) * prefix.size(), cudaMemcpyHostToDevice, st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        free_batch(b);
        delete b;
        return MR_ERR_CUDA;
    }
    *out = b;
    return MR_OK;
}

int mr_batch_run(mr_batch* b, void* stream)
{
    if (!b) return MR_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    for (const auto& g : b->groups) MR_TRY(dispatch(g.dtype, g.sigma, LaunchF{&g, st}));
    return MR_OK;
}

int mr_batch_capture(mr_batch* b, void* stream)
{
    if (!b) return MR_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    if (!st) return MR_ERR_INVALID_ARG;  // the legacy stream cannot be captured
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    MR_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int s = mr_batch_run(b, stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (s != MR_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) {
        note_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        return MR_ERR_CUDA;
    }
    b->graph = g;
    MR_CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
    return MR_OK;
}

int mr_batch_launch(mr_batch* b, void* stream)
{
    if (!b) return MR_ERR_INVALID_ARG;
    if (!b->exec) return mr_batch_run(b, stream);
    MR_CUDA_TRY(cudaGraphLaunch(b->exec, as_stream(stream)));
    return MR_OK;
}

int mr_batch_set_vectors(mr_batch* b, int32_t i, const float* x, float* y, void* stream)
{
    if (!b || i < 0 || i >= (int)b->items.size()) return MR_ERR_INVALID_ARG;
    mr_batch_item& it = b->items[(size_t)i];
    if (it.A.n_rows > 0 && (!y || (it.A.nnz > 0 && !x))) return MR_ERR_INVALID_ARG;
    it.x = x;
    it.y = y;
    Group& g = b->groups[(size_t)b->item_group[(size_t)i]];
    const int k = b->item_slot[(size_t)i];
    unsigned char* dst = g.host_ops.data() + g.op_bytes * k;
    FillF f{dst, &it.plan->p, &it.A, x, y, b->carry + b->carry_off[(size_t)i]};
    MR_TRY(dispatch(g.dtype, g.sigma, f));
    MR_CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned char*>(g.ops) + g.op_bytes * k, dst, g.op_bytes,
                                cudaMemcpyHostToDevice, as_stream(stream)));
    // the host staging slot must stay unchanged until the copy has run
    MR_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    return MR_OK;
}

int mr_batch_info(const mr_batch* b, int32_t* groups, int64_t* total_tiles)
{
    if (!b) return MR_ERR_INVALID_ARG;
    if (groups) *groups = (int32_t)b->groups.size();
    if (total_tiles) {
        long long t = 0;
        for (const auto& g : b->groups) t += g.total_tiles;
        *total_tiles = t;
    }
    return MR_OK;
}

int mr_batch_destroy(mr_batch* b)
{
    if (!b) return MR_OK;
    cudaDeviceSynchronize();
    free_batch(b);
    delete b;
    return MR_OK;
}

// ------------------------------------------------------------- autotuner ---

int mr_autotune_merbit(const mr_csr_view* A, const float* x, float* y, int32_t reps, int32_t* best_sigma,
                       int32_t* best_block, int32_t* best_flags, float* best_ms, void* stream)
{
    if (!A || !best_sigma || !best_block) return MR_ERR_INVALID_ARG;
    static const int sigmas[] = {7, 10, 14, 16, 20, 24, 28, 32};
    if (reps < 1) reps = 5;
    cudaStream_t st = as_stream(stream);
    cudaEvent_t e0, e1;
    MR_CUDA_TRY(cudaEventCreate(&e0));
    MR_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    int bs = 14, bb = 1024, bf = 0;
    int status = MR_OK;
    auto time_plan = [&](mr_merbit_plan* plan, float* out) {
        int rc = mr_spmv_merbit(plan, A, x, y, stream);  // warm
        std::vector<float> t;
        for (int r = 0; r < reps && rc == MR_OK; ++r) {
            cudaEventRecord(e0, st);
            rc = mr_spmv_merbit(plan, A, x, y, stream);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t.push_back(ms);
        }
        if (rc == MR_OK) {
            std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
            *out = t[t.size() / 2];
        }
        return rc;
    };
    for (int s : sigmas) {
        // (a) persistent kernel with its hub cache (when the plan builds one)
        mr_merbit_plan* plan = nullptr;
        status = mr_merbit_plan_create_ex(A, s, 1024, 0, stream, &plan);
        if (status != MR_OK) break;
        const bool has_hub = plan->p.hub_k > 0;
        float ms = 0.f;
        status = time_plan(plan, &ms);
        mr_merbit_plan_destroy(plan);
        if (status != MR_OK) break;
        if (ms < best) {
            best = ms;
            bs = s;
            bb = 1024;
            bf = 0;
        }
        // (b) without a hub cache, every CTA shape
        status = mr_merbit_plan_create_ex(A, s, 1024, MR_PLAN_NO_HUB_CACHE, stream, &plan);
        if (status != MR_OK) break;
        for (int blk : {128, 256, 512, 1024}) {
            if (blk == 1024 && !has_hub) continue;  // same kernel as (a)
            plan->p.block = blk;
            status = time_plan(plan, &ms);
            if (status != MR_OK) break;
            if (ms < best) {
                best = ms;
                bs = s;
                bb = blk;
                bf = MR_PLAN_NO_HUB_CACHE;
            }
        }
        mr_merbit_plan_destroy(plan);
        if (status != MR_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != MR_OK) return status;
    *best_sigma = bs;
    *best_block = bb;
    if (best_flags) *best_flags = bf;
    if (best_ms) *best_ms = best;
    return MR_OK;
}

}  // extern "C"

// Size-bucketed tuning cache: bucket = (floor(log2 rows), floor(log2 mean row
// length)); the first matrix of a bucket is tuned, later ones reuse it.
struct mr_tuner {
    std::mutex mu;
    std::map<std::pair<int, int>, std::array<int, 3>> best;  // sigma, block, flags
    int tuned = 0;
};

static std::pair<int, int> bucket_of(const mr_csr_view* A)
{
    const int r = A->n_rows > 0 ? (int)std::floor(std::log2((double)A->n_rows)) : 0;
    const double mean = A->n_rows > 0 ? (double)A->nnz / A->n_rows : 0.0;
    const int d = mean >= 1.0 ? (int)std::floor(std::log2(mean)) : 0;
    return {r, d};
}

extern "C" {

int mr_tuner_create(mr_tuner** t)
{
    if (!t) return MR_ERR_INVALID_ARG;
    *t = new (std::nothrow) mr_tuner;
    return *t ? MR_OK : MR_ERR_NOMEM;
}

int mr_tuner_destroy(mr_tuner* t)
{
    delete t;
    return MR_OK;
}

int mr_tuner_pick(mr_tuner* t, const mr_csr_view* A, const float* x, float* y, int32_t* sigma, int32_t* block,
                  int32_t* flags, void* stream)
{
    if (!t || !A || !sigma || !block) return MR_ERR_INVALID_ARG;
    const auto key = bucket_of(A);
    {
        std::lock_guard<std::mutex> lk(t->mu);
        auto f = t->best.find(key);
        if (f != t->best.end()) {
            *sigma = f->second[0];
            *block = f->second[1];
            if (flags) *flags = f->second[2];
            return MR_OK;
        }
    }
    int s = 14, b = 1024, fl = 0;
    MR_TRY(mr_autotune_merbit(A, x, y, 5, &s, &b, &fl, nullptr, stream));
    std::lock_guard<std::mutex> lk(t->mu);
    t->best[key] = {s, b, fl};
    ++t->tuned;
    *sigma = s;
    *block = b;
    if (flags) *flags = fl;
    return MR_OK;
}

int mr_tuner_stats(mr_tuner* t, int32_t* buckets, int32_t* tuned)
{
    if (!t) return MR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(t->mu);
    if (buckets) *buckets = (int32_t)t->best.size();
    if (tuned) *tuned = t->tuned;
    return MR_OK;
}

}  // extern "C"
