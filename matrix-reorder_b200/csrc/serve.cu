// Serving loop: device-resident pool of (reordered) matrices, continuous
// batching of SpMV requests, p50/p99 latency.
//
// No counterpart in the reference (a one-matrix-per-process harness).
//
//  * Pool: matrices are registered with host CSR arrays (borrowed: the caller
//    keeps them alive) and an optional permutation perm[old] = new; requests
//    then use the original numbering and the server applies x' = P x and
//    y = P^T y'. A matrix becomes resident on first use: upload + MERBIT plan
//    into stream-ordered device memory, admitted against an HBM budget, the
//    least recently used idle matrices evicted first.
//  * Streams: a three-stage pipeline in launch order: the host-to-device
//    copies of every batch on one stream, the kernels on a second, the
//    device-to-host copies on a third (event-joined per batch). The copies
//    of batch k + 1 overlap the kernels of batch k, the persistent batch
//    kernels never contend with each other for the SMs, and each batch's
//    copies run alone on their copy direction, so a batch's inputs arrive
//    as early as the link allows instead of sharing it with the batches
//    queued behind it.
//  * Batching: a scheduler thread waits `window_us` after the first pending
//    request (or until max_batch are pending), takes the pending requests in
//    arrival order, admits their matrices and launches the batch on a free
//    lane (a set of buffers and events); up to `lanes` batches are in
//    flight, so requests that arrive while others are on the GPU form the
//    next batch and overlap on the device (continuous batching). A batch is: the H2D copies of its x
//    vectors, one batched permutation, the batched MERBIT kernels (one per
//    (sigma, dtype) group; with `hub_cache`, each matrix's own persistent
//    plan with the hub cache instead, one launch per item), one batched
//    un-permutation, the D2H copies. The
//    scheduler issues a batch without holding the server lock, so submits
//    are never blocked behind the launch.
//  * Host vectors: x and y of 1 MB and more in page-locked memory
//    (cudaHostAlloc, or cudaHostRegister over the whole vector) are copied
//    by the copy engines straight from / into the caller's buffer; smaller
//    ones, and host memory that is not page-locked, go through the lane's
//    pinned staging area with a host memcpy, all of a batch's in one DMA
//    each way.
//  * Completion: a thread waits on each lane's event in launch order, copies
//    staged results to the callers' y, records latency (submit -> result in
//    y).
//  * Determinism: every request's SpMV runs the same tiles with the same
//    order of operations whatever else is in its batch, so its result is
//    bitwise the same alone and in the mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <set>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace mr;
using Clock = std::chrono::steady_clock;

namespace {

struct PermOp {
    const int32_t* perm;  // perm[old] = new, nullptr: identity
    const int32_t* n2o;   // n2o[new] = old (the inverse), nullptr: identity
    long long off;        // offset of this item's vector in the batch arena
    int n;
};

// Batched permutation of every item's vector, as a gather on both sides so
// that the writes are coalesced: inverse == 0 gives x'[j] = x[n2o[j]]
// (x' = P x), inverse != 0 gives y[i] = y'[perm[i]] (y = P^T y'). A block
// covers kPermPer * 256 consecutive elements of the batch arena, thread t
// the elements t, t + 256, ...: every thread first loads its kPermPer
// indices, then issues its kPermPer gathers, then stores, so that each
// thread has kPermPer independent loads in flight per step. A thread looks
// its item up (binary search in the prefix) for its first element and again
// only when one of its elements crosses into the next item.
constexpr int kPermPer = 8;

__global__ void __launch_bounds__(256)
    batch_permute_kernel(const PermOp* __restrict__ ops, const long long* __restrict__ prefix, int count,
                         long long total, const float* __restrict__ in, float* __restrict__ out, int inverse)
{
    const long long base = (long long)blockIdx.x * (256 * kPermPer) + threadIdx.x;
    int it = -1;
    long long lo = 0, hi = 0;
    const int32_t* idx = nullptr;
    long long src[kPermPer];
#pragma unroll
    for (int e = 0; e < kPermPer; ++e) {
        const long long g = base + 256ll * e;
        src[e] = -1;
        if (g >= total) continue;
        if (g < lo || g >= hi) {
            int a = 0, b = count - 1;  // largest item whose offset is <= g
            while (a < b) {
                const int mid = (a + b + 1) >> 1;
                if (__ldg(prefix + mid) <= g)
                    a = mid;
                else
                    b = mid - 1;
            }
            it = a;
            lo = __ldg(prefix + it);
            hi = it + 1 < count ? __ldg(prefix + it + 1) : total;
            idx = inverse ? ops[it].perm : ops[it].n2o;
        }
        src[e] = idx ? lo + __ldg(idx + (g - lo)) : g;
    }
    float v[kPermPer];
#pragma unroll
    for (int e = 0; e < kPermPer; ++e) v[e] = src[e] >= 0 ? __ldg(in + src[e]) : 0.f;
#pragma unroll
    for (int e = 0; e < kPermPer; ++e) {
        const long long g = base + 256ll * e;
        if (g < total) out[g] = v[e];
    }
}

// page-locked host memory (allocated or registered with the CUDA runtime)
bool host_pinned(const void* p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Vectors below this size move through the lane's page-locked staging
// buffers (a host memcpy into one contiguous region, then one DMA each way
// for all of them): every DMA has a fixed cost, and with both directions
// busy, a batch's small copies cut each direction's throughput by about a
// third (32 copies of log-uniform 16 KB .. 8 MB: 31 GB/s per direction;
// staging those below 256 KB: 36-39 GB/s; below 1 MB: 38-43 GB/s for 0.5-0.8
// ms of host memcpy per batch; one copy per direction: 47 GB/s). How much a
// small DMA costs varies between hosts: on a 200-matrix serving pool one
// box saturated at 15-20K req/s with 256 KB and at 24K with 1 MB.
constexpr size_t kStageBelowBytes = 1 << 20;

struct Request {
    uint64_t ticket = 0;
    int id = 0;
    const float* x = nullptr;
    float* y = nullptr;
    bool x_pinned = false, y_pinned = false;  // page-locked: copied without staging
    Clock::time_point t_submit;
    double latency_us = 0.0;
    int status = MR_OK;
    bool done = false;
};

// the request's x and y move through the staging buffers
bool item_staged(const Request& r, int32_t n)
{
    return !r.x_pinned || !r.y_pinned || sizeof(float) * (size_t)n < kStageBelowBytes;
}

struct Matrix {
    int32_t n = 0;
    int64_t nnz = 0;
    int dtype = MR_F32;
    const int32_t* h_rowptr = nullptr;
    const int32_t* h_colidx = nullptr;
    const void* h_vals = nullptr;
    const int32_t* h_perm = nullptr;
    int sigma = 14;           // MERBIT sigma of its plan
    bool persistent = false;  // single-matrix persistent plan with the hub cache, own launch
    // device state while resident
    bool resident = false;
    int refs = 0;
    uint64_t last_use = 0;
    size_t bytes = 0;
    int32_t* d_rowptr = nullptr;
    int32_t* d_colidx = nullptr;
    void* d_vals = nullptr;
    int32_t* d_perm = nullptr;
    int32_t* d_n2o = nullptr;  // inverse of d_perm, built at admission
    MerbitPlan plan;
};

template <typename T> struct PinnedVec {
    T* p = nullptr;
    size_t cap = 0;
    int reserve(size_t n)
    {
        if (n <= cap) return MR_OK;
        size_t c = std::max(n, cap * 2);
        T* q = nullptr;
        if (cudaHostAlloc(&q, sizeof(T) * c, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return MR_ERR_NOMEM;
        }
        if (p) cudaFreeHost(p);
        p = q;
        cap = c;
        return MR_OK;
    }
    ~PinnedVec()
    {
        if (p) cudaFreeHost(p);
    }
};

struct DevVec {
    void* p = nullptr;
    size_t cap = 0;  // bytes
    int reserve(size_t bytes, cudaStream_t st)
    {
        if (bytes <= cap) return MR_OK;
        size_t c = std::max(bytes, cap * 2);
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        cap = 0;
        if (cudaMallocAsync(&p, c, st) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return MR_ERR_NOMEM;
        }
        cap = c;
        return MR_OK;
    }
};

// the buffers and events of one batch in flight
struct Lane {
    cudaEvent_t done = nullptr;
    cudaEvent_t ev_start = nullptr, ev_h2d = nullptr, ev_kern = nullptr;  // stage boundaries (timing)
    PinnedVec<float> hx, hy;
    PinnedVec<unsigned char> meta_h;  // the batch's small tables, one DMA per batch
    DevVec dx, dxp, dyp, dy, carry, meta_d;
    std::vector<Request*> reqs;
    std::vector<long long> off;
    std::vector<int> mats;
    std::vector<Matrix*> mp;  // the batch's matrices, read by launch_batch without the lock
    int n_staged = 0;         // items 0 .. n_staged-1 move through hx / hy
    bool busy = false;
};

}  // namespace

struct mr_server {
    mr_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_lane;
    std::vector<std::unique_ptr<Matrix>> mats;  // stable addresses: batches read them unlocked
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, Request*> reqs;
    std::vector<Lane> lanes;
    std::deque<int> inflight;  // lane indices in launch order
    uint64_t next_ticket = 1;
    uint64_t use_clock = 0;
    size_t resident_bytes = 0;
    bool stop = false;
    std::thread sched, compl_;
    cudaStream_t admit_st = nullptr;
    cudaStream_t h2d_st = nullptr;      // the batches' host-to-device copies, in launch order
    cudaStream_t compute_st = nullptr;  // the batches' kernels, in launch order
    cudaStream_t d2h_st = nullptr;      // the batches' device-to-host copies, in launch order
    int* d_flag = nullptr;  // device word for launch_perm_invert
    int device = 0;
    // stats
    std::vector<double> lat;
    int64_t submitted = 0, completed = 0, batches = 0, admissions = 0, evictions = 0, rejected = 0, batch_items = 0;
    double t_h2d_ms = 0, t_kern_ms = 0, t_d2h_ms = 0, t_launch_ms = 0;  // summed over batches
    Clock::time_point t_first{}, t_last{};
    bool have_first = false;
    std::set<std::tuple<const void*, const void*, const void*, int32_t, int64_t>> validated;
    // page-locked or not, per host address: the driver query once per
    // address (a burst of submits would otherwise contend with the
    // scheduler's copies and launches for the driver). A stale answer only
    // changes how a vector is copied, not the result.
    std::mutex pin_mu;
    std::unordered_map<const void*, bool> pin_cache;
};

namespace {

size_t matrix_bytes(const Matrix& m)
{
    const int64_t items = (int64_t)m.n + m.nnz;
    const int64_t lanes = (items + m.sigma - 1) / m.sigma;
    const int64_t tiles = (lanes + 31) / 32;
    size_t b = sizeof(int32_t) * ((size_t)m.n + 1) + (sizeof(int32_t) + dtype_size(m.dtype)) * (size_t)m.nnz +
               (m.h_perm ? 2 * sizeof(int32_t) * (size_t)m.n : 0) + (m.sigma < 15 ? 4 : 8) * (size_t)lanes +
               8 * (size_t)(tiles + 1) + 1024;
    // the persistent plan adds the hub-remapped colidx, per-tile carries, the
    // hub column list and the per-CTA chunk tables (a bound)
    if (m.persistent) b += sizeof(int32_t) * (size_t)m.nnz + sizeof(float) * (size_t)tiles + (1u << 20);
    return b;
}

void free_resident(Matrix& m, cudaStream_t st)
{
    cudaFreeAsync(m.d_rowptr, st);
    cudaFreeAsync(m.d_colidx, st);
    cudaFreeAsync(m.d_vals, st);
    if (m.d_perm) cudaFreeAsync(m.d_perm, st);
    if (m.d_n2o) cudaFreeAsync(m.d_n2o, st);
    cudaFreeAsync(m.plan.tile_x, st);
    cudaFreeAsync(m.plan.tile_y, st);
    cudaFreeAsync(m.plan.lane_desc, st);
    // the persistent plan's own buffers (cudaMalloc'd by the plan builders);
    // the matrix is idle, its last batch retired
    for (void* q : {(void*)m.plan.carry, (void*)m.plan.ticket, (void*)m.plan.colh, (void*)m.plan.hub_cols,
                    (void*)m.plan.chunk_start, (void*)m.plan.boundary_run, (void*)m.plan.boundary_flag})
        if (q) cudaFree(q);
    m.plan = MerbitPlan();
    m.d_rowptr = m.d_colidx = m.d_perm = m.d_n2o = nullptr;
    m.d_vals = nullptr;
    m.plan.tile_x = m.plan.tile_y = nullptr;
    m.plan.lane_desc = nullptr;
    m.resident = false;
}

// upload + plan on the admission stream (called with the server lock held)
int make_resident(mr_server* s, Matrix& m)
{
    cudaStream_t st = s->admit_st;
    const size_t vb = dtype_size(m.dtype);
    auto alloc = [&](void** p, size_t b) { return cudaMallocAsync(p, std::max<size_t>(b, 16), st) == cudaSuccess; };
    m.plan = MerbitPlan();
    m.plan.sigma = m.sigma;
    m.plan.block = 256;
    cudaGetDevice(&m.plan.device);
    m.plan.n_rows = m.n;
    m.plan.nnz = m.nnz;
    const int64_t items = (int64_t)m.n + m.nnz;
    m.plan.lane_num = (int)((items + m.plan.sigma - 1) / m.plan.sigma);
    m.plan.tile_num = (m.plan.lane_num + 31) / 32;
    const size_t desc_b = m.plan.sigma < 15 ? 4 : 8;
    bool ok = alloc((void**)&m.d_rowptr, 4 * ((size_t)m.n + 1)) && alloc((void**)&m.d_colidx, 4 * (size_t)m.nnz) &&
              alloc(&m.d_vals, vb * (size_t)m.nnz) && (!m.h_perm || (alloc((void**)&m.d_perm, 4 * (size_t)m.n) && alloc((void**)&m.d_n2o, 4 * (size_t)m.n))) &&
              alloc((void**)&m.plan.tile_x, 4 * ((size_t)m.plan.tile_num + 1)) &&
              alloc((void**)&m.plan.tile_y, 4 * ((size_t)m.plan.tile_num + 1)) &&
              alloc(&m.plan.lane_desc, desc_b * (size_t)std::max(m.plan.lane_num, 1));
    if (!ok) {
        cudaGetLastError();
        free_resident(m, st);
        return MR_ERR_NOMEM;
    }
    cudaMemcpyAsync(m.d_rowptr, m.h_rowptr, 4 * ((size_t)m.n + 1), cudaMemcpyHostToDevice, st);
    if (m.nnz > 0) {
        cudaMemcpyAsync(m.d_colidx, m.h_colidx, 4 * (size_t)m.nnz, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(m.d_vals, m.h_vals, vb * (size_t)m.nnz, cudaMemcpyHostToDevice, st);
    }
    int rc0 = MR_OK;
    if (m.h_perm) {
        cudaMemcpyAsync(m.d_perm, m.h_perm, 4 * (size_t)m.n, cudaMemcpyHostToDevice, st);
        // the permutation was checked on the host at registration; the flag only satisfies the kernel
        rc0 = launch_perm_invert(m.n, m.d_perm, m.d_n2o, s->d_flag, st);
    }
    int rc = rc0 != MR_OK ? rc0
                          : launch_merbit_plan(m.d_rowptr, m.n, (int)m.nnz, m.plan.sigma, m.plan.lane_num,
                                               m.plan.tile_num, m.plan.tile_x, m.plan.tile_y, m.plan.lane_desc, st);
    if (rc == MR_OK && m.persistent) {
        // the single-matrix persistent plan: carries, completion ticket, hub
        // cache and cost-balanced CTA chunks, as mr_merbit_plan_create builds
        m.plan.block = 1024;
        if (cudaMalloc(&m.plan.carry, sizeof(float) * (size_t)std::max(m.plan.tile_num, 1)) != cudaSuccess ||
            cudaMalloc(&m.plan.ticket, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            rc = MR_ERR_NOMEM;
        } else if (cudaMemsetAsync(m.plan.ticket, 0, sizeof(int), st) != cudaSuccess) {
            rc = MR_ERR_CUDA;
        } else {
            const mr_csr_view A{m.n, m.n, m.nnz, m.d_rowptr, m.d_colidx, m.d_vals, m.dtype};
            rc = build_hub_cache(m.plan, A, st);
            if (rc == MR_OK) rc = build_chunk_bounds(m.plan, m.d_colidx, st);
        }
    }
    if (rc == MR_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = MR_ERR_CUDA;
    if (rc != MR_OK) {
        free_resident(m, st);
        return rc;
    }
    m.resident = true;
    m.bytes = matrix_bytes(m);
    return MR_OK;
}

// make room for `need` bytes by evicting least recently used idle matrices
bool make_room(mr_server* s, size_t need, const std::vector<int>& keep)
{
    while (s->resident_bytes + need > (size_t)s->cfg.hbm_budget_bytes) {
        int victim = -1;
        for (int i = 0; i < (int)s->mats.size(); ++i) {
            const Matrix& m = *s->mats[(size_t)i];
            if (!m.resident || m.refs > 0) continue;
            if (std::find(keep.begin(), keep.end(), i) != keep.end()) continue;
            if (victim < 0 || m.last_use < s->mats[(size_t)victim]->last_use) victim = i;
        }
        if (victim < 0) return false;
        Matrix& v = *s->mats[(size_t)victim];
        free_resident(v, s->admit_st);
        s->resident_bytes -= v.bytes;
        ++s->evictions;
    }
    return true;
}

int launch_batch(mr_server* s, Lane& L)
{
    const int count = (int)L.reqs.size();
    // staged items (small vectors, or a vector not page-locked) go first, so
    // that they form one contiguous region of the arena and of the staging
    // buffers: one DMA each way for all of them
    {
        std::vector<int> order((size_t)count);
        for (int i = 0; i < count; ++i) order[(size_t)i] = i;
        auto staged_item = [&](int i) { return item_staged(*L.reqs[(size_t)i], L.mp[(size_t)i]->n); };
        std::stable_partition(order.begin(), order.end(), staged_item);
        std::vector<Request*> reqs((size_t)count);
        std::vector<int> mats((size_t)count);
        std::vector<Matrix*> mp((size_t)count);
        for (int i = 0; i < count; ++i) {
            const int o = order[(size_t)i];
            reqs[(size_t)i] = L.reqs[(size_t)o];
            mats[(size_t)i] = L.mats[(size_t)o];
            mp[(size_t)i] = L.mp[(size_t)o];
        }
        L.reqs.swap(reqs);
        L.mats.swap(mats);
        L.mp.swap(mp);
    }
    L.off.assign((size_t)count + 1, 0);
    L.n_staged = 0;
    for (int i = 0; i < count; ++i) {
        L.off[(size_t)i + 1] = L.off[(size_t)i] + L.mp[(size_t)i]->n;
        if (item_staged(*L.reqs[(size_t)i], L.mp[(size_t)i]->n)) L.n_staged = i + 1;
    }
    const long long total = L.off[(size_t)count];
    const long long staged_elems = L.off[(size_t)L.n_staged];
    if (staged_elems > 0) {
        MR_TRY(L.hx.reserve((size_t)staged_elems));
        MR_TRY(L.hy.reserve((size_t)staged_elems));
    }
    for (int i = 0; i < L.n_staged; ++i)
        std::memcpy(L.hx.p + L.off[(size_t)i], L.reqs[(size_t)i]->x,
                    sizeof(float) * (size_t)(L.off[(size_t)i + 1] - L.off[(size_t)i]));
    const size_t vbytes = sizeof(float) * (size_t)(total + 1);
    // a lane's buffers are (re)allocated in the order of the copy stream
    // that first writes them; the lane is idle (its last batch completed)
    cudaStream_t st = s->h2d_st;
    MR_TRY(L.dx.reserve(vbytes, st));
    MR_TRY(L.dxp.reserve(vbytes, st));
    MR_TRY(L.dyp.reserve(vbytes, st));
    MR_TRY(L.dy.reserve(vbytes, st));
    // group the items by (sigma, dtype): one batched kernel per group; items
    // with a persistent plan run alone, one launch each
    std::map<std::pair<int, int>, std::vector<int>> groups;
    std::vector<int> solo;
    long long carry_total = 0;
    std::vector<long long> carry_off((size_t)count);
    for (int i = 0; i < count; ++i) {
        const Matrix& m = *L.mp[(size_t)i];
        if (m.persistent)
            solo.push_back(i);
        else
            groups[{m.plan.sigma, m.dtype}].push_back(i);
        carry_off[(size_t)i] = carry_total;
        carry_total += std::max(m.plan.tile_num, 1);
    }
    MR_TRY(L.carry.reserve(sizeof(float) * (size_t)carry_total, st));
    // the small tables (batch operands per group, tile prefixes, permutation
    // operands) live in one pinned block per lane and go over in one copy:
    // a pageable source could make the copy wait for the lane's stream
    auto a256 = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t ops_bytes = 0;
    for (auto& g : groups) ops_bytes += a256(batch_op_bytes(g.first.second, g.first.first) * g.second.size());
    const size_t at_prefix = ops_bytes;
    const size_t at_pops = at_prefix + a256(sizeof(long long) * ((size_t)count + groups.size()));
    const size_t at_pprefix = at_pops + a256(sizeof(PermOp) * (size_t)count);
    const size_t meta_bytes = at_pprefix + sizeof(long long) * ((size_t)count + 1);
    MR_TRY(L.meta_h.reserve(meta_bytes));
    MR_TRY(L.meta_d.reserve(meta_bytes, st));
    unsigned char* mh = L.meta_h.p;
    unsigned char* md = static_cast<unsigned char*>(L.meta_d.p);
    long long* prefix_host = reinterpret_cast<long long*>(mh + at_prefix);
    size_t n_prefix = 0;
    PermOp* pops = reinterpret_cast<PermOp*>(mh + at_pops);
    float* dx = static_cast<float*>(L.dx.p);
    float* dxp = static_cast<float*>(L.dxp.p);
    float* dyp = static_cast<float*>(L.dyp.p);
    float* dy = static_cast<float*>(L.dy.p);
    float* carry = static_cast<float*>(L.carry.p);
    struct GroupLaunch {
        int dtype, sigma, count;
        size_t ops_at, prefix_at;
        long long tiles;
    };
    std::vector<GroupLaunch> gl;
    size_t at = 0;
    for (auto& g : groups) {
        const int sigma = g.first.first, dtype = g.first.second;
        const size_t ob = batch_op_bytes(dtype, sigma);
        GroupLaunch x{dtype, sigma, (int)g.second.size(), at, n_prefix, 0};
        prefix_host[n_prefix++] = 0;
        for (int i : g.second) {
            const Matrix& m = *L.mp[(size_t)i];
            const mr_csr_view A{m.n, m.n, m.nnz, m.d_rowptr, m.d_colidx, m.d_vals, m.dtype};
            MR_TRY(batch_fill_op(mh + at, dtype, sigma, m.plan, A, dxp + L.off[(size_t)i], dyp + L.off[(size_t)i],
                                 carry + carry_off[(size_t)i]));
            at += ob;
            x.tiles += m.plan.tile_num;
            prefix_host[n_prefix++] = x.tiles;
        }
        at = (at + 255) / 256 * 256;
        gl.push_back(x);
    }
    for (int i = 0; i < count; ++i) {
        const Matrix& m = *L.mp[(size_t)i];
        pops[(size_t)i] = PermOp{m.d_perm, m.d_n2o, L.off[(size_t)i], m.n};
    }
    std::memcpy(mh + at_pprefix, L.off.data(), sizeof(long long) * ((size_t)count + 1));
    MR_CUDA_TRY(cudaEventRecord(L.ev_start, st));
    MR_CUDA_TRY(cudaMemcpyAsync(md, mh, meta_bytes, cudaMemcpyHostToDevice, st));
    if (staged_elems > 0)
        MR_CUDA_TRY(cudaMemcpyAsync(dx, L.hx.p, sizeof(float) * (size_t)staged_elems, cudaMemcpyHostToDevice, st));
    for (int i = L.n_staged; i < count; ++i) {
        const size_t o = (size_t)L.off[(size_t)i], nb = sizeof(float) * ((size_t)L.off[(size_t)i + 1] - o);
        MR_CUDA_TRY(cudaMemcpyAsync(dx + o, L.reqs[(size_t)i]->x, nb, cudaMemcpyHostToDevice, st));
    }
    MR_CUDA_TRY(cudaEventRecord(L.ev_h2d, st));
    st = s->compute_st;
    MR_CUDA_TRY(cudaStreamWaitEvent(st, L.ev_h2d, 0));
    const int pgrid = (int)std::max<long long>(1, (total + 256 * kPermPer - 1) / (256 * kPermPer));
    const PermOp* d_pops = reinterpret_cast<const PermOp*>(md + at_pops);
    const long long* d_pprefix = reinterpret_cast<const long long*>(md + at_pprefix);
    batch_permute_kernel<<<pgrid, 256, 0, st>>>(d_pops, d_pprefix, count, total, dx, dxp, 0);
    MR_CUDA_TRY(cudaGetLastError());
    for (const auto& g : gl)
        MR_TRY(batch_launch_ops(g.dtype, g.sigma, md + g.ops_at,
                                reinterpret_cast<const long long*>(md + at_prefix) + g.prefix_at, g.count, g.tiles,
                                st));
    // one plan's launches never overlap: they are ordered on this stream
    for (int i : solo) {
        const Matrix& m = *L.mp[(size_t)i];
        MR_TRY(launch_merbit_spmv(m.plan, m.d_colidx, m.d_vals, m.dtype, dxp + L.off[(size_t)i],
                                  dyp + L.off[(size_t)i], m.plan.carry, st));
    }
    batch_permute_kernel<<<pgrid, 256, 0, st>>>(d_pops, d_pprefix, count, total, dyp, dy, 1);
    MR_CUDA_TRY(cudaGetLastError());
    MR_CUDA_TRY(cudaEventRecord(L.ev_kern, st));
    st = s->d2h_st;
    MR_CUDA_TRY(cudaStreamWaitEvent(st, L.ev_kern, 0));
    if (staged_elems > 0)
        MR_CUDA_TRY(cudaMemcpyAsync(L.hy.p, dy, sizeof(float) * (size_t)staged_elems, cudaMemcpyDeviceToHost, st));
    for (int i = L.n_staged; i < count; ++i) {
        const size_t o = (size_t)L.off[(size_t)i], nb = sizeof(float) * ((size_t)L.off[(size_t)i + 1] - o);
        MR_CUDA_TRY(cudaMemcpyAsync(L.reqs[(size_t)i]->y, dy + o, nb, cudaMemcpyDeviceToHost, st));
    }
    MR_CUDA_TRY(cudaEventRecord(L.done, st));
    return MR_OK;
}

void finish_requests(mr_server* s, std::vector<Request*>& rs, int status)
{
    const auto now = Clock::now();
    for (Request* r : rs) {
        r->status = status;
        r->latency_us = std::chrono::duration<double, std::micro>(now - r->t_submit).count();
        r->done = true;
        if (status == MR_OK) {
            s->lat.push_back(r->latency_us);
            ++s->completed;
        } else {
            ++s->rejected;
        }
    }
    s->t_last = now;
}

void scheduler_loop(mr_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_sched.wait(lk, [&] { return s->stop || !s->pending.empty(); });
        if (s->stop) return;
        // batching window: from the first pending request's arrival
        const auto deadline = s->pending.front()->t_submit + std::chrono::microseconds(s->cfg.window_us);
        s->cv_sched.wait_until(lk, deadline, [&] { return s->stop || (int)s->pending.size() >= s->cfg.max_batch; });
        if (s->stop) return;
        int lane = -1;
        s->cv_lane.wait(lk, [&] {
            if (s->stop) return true;
            for (int i = 0; i < (int)s->lanes.size(); ++i)
                if (!s->lanes[(size_t)i].busy) {
                    lane = i;
                    return true;
                }
            return false;
        });
        if (s->stop) return;
        Lane& L = s->lanes[(size_t)lane];
        L.reqs.clear();
        L.mats.clear();
        L.mp.clear();
        std::vector<int> keep;
        std::deque<Request*> deferred;
        while (!s->pending.empty() && (int)L.reqs.size() < s->cfg.max_batch) {
            Request* r = s->pending.front();
            s->pending.pop_front();
            Matrix& m = *s->mats[(size_t)r->id];
            if (!m.resident) {
                const size_t need = matrix_bytes(m);
                if (need > (size_t)s->cfg.hbm_budget_bytes) {  // can never fit
                    std::vector<Request*> one{r};
                    finish_requests(s, one, MR_ERR_BUSY);
                    continue;
                }
                if (!make_room(s, need, keep)) {  // all room is pinned by batches in flight
                    deferred.push_back(r);
                    continue;
                }
                const int rc = make_resident(s, m);
                if (rc != MR_OK) {
                    std::vector<Request*> one{r};
                    finish_requests(s, one, rc);
                    continue;
                }
                s->resident_bytes += m.bytes;
                ++s->admissions;
            }
            m.last_use = ++s->use_clock;
            ++m.refs;
            keep.push_back(r->id);
            L.reqs.push_back(r);
            L.mats.push_back(r->id);
            L.mp.push_back(&m);
        }
        for (auto it = deferred.rbegin(); it != deferred.rend(); ++it) s->pending.push_front(*it);
        if (L.reqs.empty()) {
            // everything deferred: wait for a batch to finish and free room
            s->cv_done.wait_for(lk, std::chrono::milliseconds(1));
            continue;
        }
        L.busy = true;
        lk.unlock();
        const auto tl = Clock::now();
        const int rc = launch_batch(s, L);
        const double launch_ms = std::chrono::duration<double, std::milli>(Clock::now() - tl).count();
        lk.lock();
        s->t_launch_ms += launch_ms;
        if (rc != MR_OK) {
            for (int id : L.mats) --s->mats[(size_t)id]->refs;
            finish_requests(s, L.reqs, rc);
            L.busy = false;
            s->cv_done.notify_all();
            continue;
        }
        ++s->batches;
        s->batch_items += (int64_t)L.reqs.size();
        s->inflight.push_back(lane);
        s->cv_done.notify_all();  // wakes the completion thread
    }
}

void completion_loop(mr_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_done.wait(lk, [&] { return s->stop || !s->inflight.empty(); });
        if (s->inflight.empty() && s->stop) return;
        const int lane = s->inflight.front();
        Lane& L = s->lanes[(size_t)lane];
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(L.done);
        float t_h2d = 0.f, t_kern = 0.f, t_d2h = 0.f;
        if (e == cudaSuccess) {
            cudaEventElapsedTime(&t_h2d, L.ev_start, L.ev_h2d);
            cudaEventElapsedTime(&t_kern, L.ev_h2d, L.ev_kern);
            cudaEventElapsedTime(&t_d2h, L.ev_kern, L.done);
        }
        // results to the callers' buffers
        if (e == cudaSuccess)
            for (size_t i = 0; i < (size_t)L.n_staged; ++i)
                std::memcpy(L.reqs[i]->y, L.hy.p + L.off[i], sizeof(float) * (size_t)(L.off[i + 1] - L.off[i]));
        lk.lock();
        s->t_h2d_ms += t_h2d;
        s->t_kern_ms += t_kern;
        s->t_d2h_ms += t_d2h;
        s->inflight.pop_front();
        for (int id : L.mats) --s->mats[(size_t)id]->refs;
        finish_requests(s, L.reqs, e == cudaSuccess ? MR_OK : MR_ERR_CUDA);
        L.reqs.clear();
        L.busy = false;
        s->cv_done.notify_all();
        s->cv_lane.notify_all();
        s->cv_sched.notify_all();
    }
}

}  // namespace

namespace {

bool pinned_cached(mr_server* s, const void* p)
{
    {
        std::lock_guard<std::mutex> lk(s->pin_mu);
        auto it = s->pin_cache.find(p);
        if (it != s->pin_cache.end()) return it->second;
    }
    const bool v = host_pinned(p);
    std::lock_guard<std::mutex> lk(s->pin_mu);
    if (s->pin_cache.size() >= 65536) s->pin_cache.clear();
    s->pin_cache[p] = v;
    return v;
}

}  // namespace

extern "C" {

int mr_server_create(const mr_server_config* cfg, mr_server** out)
{
    if (!out) return MR_ERR_INVALID_ARG;
    *out = nullptr;
    auto* s = new (std::nothrow) mr_server;
    if (!s) return MR_ERR_NOMEM;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.window_us <= 0) s->cfg.window_us = 200;
    if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
    if (s->cfg.lanes <= 0) s->cfg.lanes = 3;
    if (s->cfg.sigma <= 0) s->cfg.sigma = 14;
    if (!merbit_sigma_supported(s->cfg.sigma) || s->cfg.lanes > 16) {
        delete s;
        return MR_ERR_INVALID_ARG;
    }
    cudaGetDevice(&s->device);
    if (s->cfg.hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        s->cfg.hbm_budget_bytes = (int64_t)(fr / 2);
    }
    s->lanes.resize((size_t)s->cfg.lanes);
    bool ok = cudaStreamCreateWithFlags(&s->admit_st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->h2d_st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->compute_st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->d2h_st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&s->d_flag, sizeof(int)) == cudaSuccess &&
              cudaMemset(s->d_flag, 0, sizeof(int)) == cudaSuccess;
    for (auto& L : s->lanes)
        ok = ok && cudaEventCreate(&L.done) == cudaSuccess && cudaEventCreate(&L.ev_start) == cudaSuccess &&
             cudaEventCreate(&L.ev_h2d) == cudaSuccess && cudaEventCreate(&L.ev_kern) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        mr_server_destroy(s);
        return MR_ERR_CUDA;
    }
    s->sched = std::thread(scheduler_loop, s);
    s->compl_ = std::thread(completion_loop, s);
    *out = s;
    return MR_OK;
}

int mr_server_add_matrix(mr_server* s, int32_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx,
                         const void* vals, int32_t dtype, const int32_t* perm_old2new, int32_t* id)
{
    if (!s || !id || n <= 0 || nnz < 0 || nnz > INT32_MAX || !rowptr || (nnz > 0 && (!colidx || !vals)))
        return MR_ERR_INVALID_ARG;
    if (dtype != MR_F32 && dtype != MR_F16 && dtype != MR_BF16) return MR_ERR_UNSUPPORTED;
    // host-side validation (the pool admits matrices without a device
    // check); arrays already validated for an earlier registration are not
    // scanned again (the caller keeps registered arrays unchanged)
    const auto key = std::make_tuple((const void*)rowptr, (const void*)colidx, (const void*)perm_old2new, n, nnz);
    bool known;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        known = s->validated.count(key) > 0;
    }
    if (!known) {
        if (rowptr[0] != 0 || rowptr[n] != nnz) return MR_ERR_INVALID_ARG;
        for (int32_t i = 0; i < n; ++i)
            if (rowptr[i + 1] < rowptr[i]) return MR_ERR_INVALID_ARG;
        for (int64_t k = 0; k < nnz; ++k)
            if (colidx[k] < 0 || colidx[k] >= n) return MR_ERR_INVALID_ARG;
        if (perm_old2new) {
            std::vector<char> seen((size_t)n, 0);
            for (int32_t i = 0; i < n; ++i) {
                const int32_t p = perm_old2new[i];
                if (p < 0 || p >= n || seen[(size_t)p]) return MR_ERR_INVALID_PERM;
                seen[(size_t)p] = 1;
            }
        }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->validated.insert(key);
    Matrix m;
    m.n = n;
    m.nnz = nnz;
    m.dtype = dtype;
    m.h_rowptr = rowptr;
    m.h_colidx = colidx;
    m.h_vals = vals;
    m.h_perm = perm_old2new;
    m.sigma = s->cfg.sigma;
    m.persistent = s->cfg.hub_cache != 0;
    auto pm = std::unique_ptr<Matrix>(new (std::nothrow) Matrix(m));
    if (!pm) return MR_ERR_NOMEM;
    s->mats.push_back(std::move(pm));
    *id = (int32_t)s->mats.size() - 1;
    return MR_OK;
}

int mr_server_submit(mr_server* s, int32_t id, const float* x, float* y, uint64_t* ticket)
{
    if (!s || !x || !y) return MR_ERR_INVALID_ARG;
    auto* r = new (std::nothrow) Request;
    if (!r) return MR_ERR_NOMEM;
    r->id = id;
    r->x = x;
    r->y = y;
    r->x_pinned = pinned_cached(s, x);
    r->y_pinned = pinned_cached(s, y);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (id < 0 || id >= (int)s->mats.size()) {
            delete r;
            return MR_ERR_NOT_FOUND;
        }
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->pending.push_back(r);
        ++s->submitted;
        if (!s->have_first) {
            s->t_first = r->t_submit;
            s->have_first = true;
        }
    }
    s->cv_sched.notify_one();
    if (ticket) *ticket = r->ticket;
    return MR_OK;
}

int mr_server_wait(mr_server* s, uint64_t ticket, int32_t timeout_ms, double* latency_us)
{
    if (!s) return MR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return MR_ERR_NOT_FOUND;
    Request* r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                                        [&] { return r->done; });
    if (!ok) return MR_ERR_TIMEOUT;
    const int st = r->status;
    if (latency_us) *latency_us = r->latency_us;
    s->reqs.erase(it);
    delete r;
    return st;
}

int mr_server_drain(mr_server* s, int32_t timeout_ms)
{
    if (!s) return MR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms), [&] {
        return s->pending.empty() && s->inflight.empty() && s->completed + s->rejected == s->submitted;
    });
    // forget finished requests nobody waits for
    for (auto it = s->reqs.begin(); it != s->reqs.end();) {
        if (it->second->done) {
            delete it->second;
            it = s->reqs.erase(it);
        } else {
            ++it;
        }
    }
    return ok ? MR_OK : MR_ERR_TIMEOUT;
}

int mr_server_get_stats(mr_server* s, mr_server_stats* out)
{
    if (!s || !out) return MR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    mr_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.rejected = s->rejected;
    st.batches = s->batches;
    st.admissions = s->admissions;
    st.evictions = s->evictions;
    st.resident_bytes = (int64_t)s->resident_bytes;
    int64_t nres = 0;
    for (const auto& m : s->mats) nres += m->resident ? 1 : 0;
    st.resident_matrices = nres;
    st.mean_batch = s->batches ? (double)s->batch_items / (double)s->batches : 0.0;
    st.h2d_ms = s->t_h2d_ms;
    st.compute_ms = s->t_kern_ms;
    st.d2h_ms = s->t_d2h_ms;
    st.launch_ms = s->t_launch_ms;
    if (!s->lat.empty()) {
        std::vector<double> v = s->lat;
        auto pct = [&](double q) {
            const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + (long)k, v.end());
            return v[k];
        };
        st.p50_us = pct(0.50);
        st.p99_us = pct(0.99);
        double sum = 0, mx = 0;
        for (double d : s->lat) {
            sum += d;
            mx = std::max(mx, d);
        }
        st.mean_us = sum / (double)s->lat.size();
        st.max_us = mx;
        const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        st.req_per_s = span > 0 ? (double)s->completed / span : 0.0;
    }
    *out = st;
    return MR_OK;
}

int mr_server_reset_stats(mr_server* s)
{
    if (!s) return MR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat.clear();
    s->submitted -= s->completed + s->rejected;
    s->completed = s->rejected = s->batches = s->batch_items = 0;
    s->t_h2d_ms = s->t_kern_ms = s->t_d2h_ms = s->t_launch_ms = 0;
    s->admissions = s->evictions = 0;
    s->have_first = false;
    return MR_OK;
}

int mr_server_destroy(mr_server* s)
{
    if (!s) return MR_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_sched.notify_all();
    s->cv_lane.notify_all();
    s->cv_done.notify_all();
    if (s->sched.joinable()) s->sched.join();
    if (s->compl_.joinable()) s->compl_.join();
    cudaDeviceSynchronize();
    for (auto& m : s->mats)
        if (m->resident) free_resident(*m, s->admit_st);
    for (auto& L : s->lanes) {
        for (DevVec* d : {&L.dx, &L.dxp, &L.dyp, &L.dy, &L.carry, &L.meta_d})
            if (d->p) cudaFreeAsync(d->p, s->admit_st);
        for (cudaEvent_t ev : {L.done, L.ev_start, L.ev_h2d, L.ev_kern})
            if (ev) cudaEventDestroy(ev);
    }
    if (s->admit_st) {
        cudaStreamSynchronize(s->admit_st);
        cudaStreamDestroy(s->admit_st);
    }
    if (s->d_flag) cudaFree(s->d_flag);
    for (cudaStream_t st : {s->h2d_st, s->compute_st, s->d2h_st})
        if (st) cudaStreamDestroy(st);
    for (auto& kv : s->reqs) delete kv.second;
    for (Request* r : s->pending)
        if (s->reqs.find(r->ticket) == s->reqs.end()) delete r;
    delete s;
    return MR_OK;
}

// Open-loop Poisson load: n_requests arrivals at `rate` per second, matrix
// ids drawn uniformly from ids[], x / y buffers per id (y buffers are
// overwritten by every request of that id). Returns after all completed.
int mr_server_loadgen(mr_server* s, const int32_t* ids, int32_t n_ids, int64_t n_requests, double rate,
                      uint64_t seed, const float* const* x_of, float* const* y_of, int32_t timeout_ms)
{
    if (!s || !ids || n_ids <= 0 || n_requests < 0 || rate <= 0 || !x_of || !y_of) return MR_ERR_INVALID_ARG;
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate);
    std::uniform_int_distribution<int> pick(0, n_ids - 1);
    auto t = Clock::now();
    for (int64_t i = 0; i < n_requests; ++i) {
        t += std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(gap(rng)));
        while (Clock::now() < t) {
            // spin: arrivals are tens of microseconds apart
        }
        const int k = pick(rng);
        MR_TRY(mr_server_submit(s, ids[k], x_of[k], y_of[k], nullptr));
    }
    return mr_server_drain(s, timeout_ms);
}

// Plain per-request path (the comparison baseline for the server): each
// request in turn copies x to the device, permutes it, runs one MERBIT SpMV
// with its own plan, un-permutes y, copies it back and synchronises. Host
// vectors follow the server's rule: page-locked ones are copied directly,
// others through a pinned staging buffer.
int mr_plain_requests(int32_t n_mats, const mr_merbit_plan* const* plans, const mr_csr_view* views,
                      const int32_t* const* perm_dev, int64_t n_requests, const int32_t* req_mat,
                      const float* const* x_host, float* const* y_host, void* stream, double* elapsed_ms,
                      double* lat_us)
{
    if (n_mats <= 0 || !plans || !views || !perm_dev || n_requests < 0 || !req_mat || !x_host || !y_host)
        return MR_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    int32_t nmax = 0;
    for (int i = 0; i < n_mats; ++i) {
        if (!plans[i] || views[i].n_rows != views[i].n_cols) return MR_ERR_INVALID_ARG;
        nmax = std::max(nmax, views[i].n_rows);
    }
    for (int64_t r = 0; r < n_requests; ++r)
        if (req_mat[r] < 0 || req_mat[r] >= n_mats || !x_host[r] || !y_host[r]) return MR_ERR_INVALID_ARG;
    PinnedVec<float> hx, hy;
    MR_TRY(hx.reserve((size_t)nmax + 1));
    MR_TRY(hy.reserve((size_t)nmax + 1));
    DevBuf dx, dxp, dyp, dy;
    MR_TRY(dx.alloc(sizeof(float) * ((size_t)nmax + 1), st));
    MR_TRY(dxp.alloc(sizeof(float) * ((size_t)nmax + 1), st));
    MR_TRY(dyp.alloc(sizeof(float) * ((size_t)nmax + 1), st));
    MR_TRY(dy.alloc(sizeof(float) * ((size_t)nmax + 1), st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    const auto t0 = Clock::now();
    for (int64_t r = 0; r < n_requests; ++r) {
        const auto tr = Clock::now();
        const int k = req_mat[r];
        const int n = views[k].n_rows;
        const size_t nb = sizeof(float) * (size_t)n;
        const bool xp = host_pinned(x_host[r]), yp = host_pinned(y_host[r]);
        if (!xp) std::memcpy(hx.p, x_host[r], nb);
        MR_CUDA_TRY(cudaMemcpyAsync(dx.p, xp ? x_host[r] : hx.p, nb, cudaMemcpyHostToDevice, st));
        MR_TRY(launch_permute_vector(n, perm_dev[k], dx.as<float>(), dxp.as<float>(), 0, st));
        MR_TRY(mr_spmv_merbit(plans[k], &views[k], dxp.as<float>(), dyp.as<float>(), stream));
        MR_TRY(launch_permute_vector(n, perm_dev[k], dyp.as<float>(), dy.as<float>(), 1, st));
        MR_CUDA_TRY(cudaMemcpyAsync(yp ? y_host[r] : hy.p, dy.p, nb, cudaMemcpyDeviceToHost, st));
        MR_CUDA_TRY(cudaStreamSynchronize(st));
        if (!yp) std::memcpy(y_host[r], hy.p, nb);
        if (lat_us) lat_us[r] = std::chrono::duration<double, std::micro>(Clock::now() - tr).count();
    }
    if (elapsed_ms) *elapsed_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    return MR_OK;
}

}  // extern "C"
