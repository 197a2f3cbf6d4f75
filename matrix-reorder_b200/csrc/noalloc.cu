// Allocation-free MERBIT SpMV: plan, carries and flags live in one
// file-scope device array, so a call performs no device allocation at all.
//
// Who needs it: callers that must not allocate device memory while they run
// SpMV — code that owns the whole device heap through its own pool (a
// serving runtime, another framework's caching allocator), code running in
// a context where cudaMalloc / cudaFree would synchronise the device or is
// forbidden (a latency-critical loop, a real-time thread), and embedded
// users that budget device memory up front. They still pass the matrix, x
// and y; everything else comes from the static array.
//
// Limits and rules:
//  * the array holds the plan of at most kNoAllocMaxItems merge items
//    (n_rows + nnz <= 2^24) with SIGMA 14, about 5.3 MB that every GPU which
//    loads the library keeps until the process exits; larger matrices get
//    MR_ERR_UNSUPPORTED before any work is enqueued;
//  * each call first checks the matrix as plan creation does (rowptr
//    starts at 0, never decreases and ends at nnz; every column index lies
//    in [0, n_cols)), with the check's flag in the array, and waits for the
//    answer on the caller's stream: a malformed matrix returns
//    MR_ERR_INVALID_ARG before any gather is issued;
//  * it then rebuilds the plan into the array (one extra kernel) and runs
//    the same persistent MERBIT kernel as mr_spmv_merbit, so results are
//    bitwise those of a planned call;
//  * the first call on a device does a set-up: it looks up the array's
//    device address (cudaGetSymbolAddress, with that device current) and
//    keeps it for the process, so that first call should come before any
//    stream capture. The kept address dies with the device's context: after
//    cudaDeviceReset the entry point must not be called again in that
//    process;
//  * all calls share the array and it keeps the last call's contents, so
//    calls whose work overlaps on the GPU (different streams, or threads
//    without ordering) race: serialise them on one stream. Every call
//    rewrites the plan and the carries before reading them, and clears the
//    check flag and the completion ticket of the persistent kernel (the
//    words that must start at zero) with cudaMemsetAsync, which allocates
//    nothing.
#include <mutex>

#include "common.cuh"
#include "internal.hpp"

namespace mr {
namespace {

constexpr int kNoAllocSigma = 14;
constexpr long long kNoAllocMaxItems = 1ll << 24;
constexpr long long kNoAllocMaxLanes = (kNoAllocMaxItems + kNoAllocSigma - 1) / kNoAllocSigma;
constexpr long long kNoAllocMaxTiles = (kNoAllocMaxLanes + 31) / 32;
// tile_x, tile_y (tiles + 1 each), lane descriptors, carries; 256-byte slots
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffTileX = 0;
constexpr size_t kOffTileY = kOffTileX + align256(4 * (kNoAllocMaxTiles + 1));
constexpr size_t kOffDesc = kOffTileY + align256(4 * (kNoAllocMaxTiles + 1));
constexpr size_t kOffCarry = kOffDesc + align256(4 * kNoAllocMaxLanes);
constexpr size_t kOffTicket = kOffCarry + align256(4 * kNoAllocMaxTiles);
constexpr size_t kOffFlag = kOffTicket + 128;  // validation flag, same 256-byte slot
constexpr size_t kNoAllocBytes = kOffTicket + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_mu;
void* g_addr[64] = {};

int scratch_address(void** out)
{
    int dev = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return MR_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        MR_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return MR_OK;
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" int mr_spmv_merbit_noalloc(const mr_csr_view* A, const float* x, float* y, void* stream)
{
    if (!A || A->n_rows < 0 || A->n_cols < 0 || A->nnz < 0 || !A->rowptr) return MR_ERR_INVALID_ARG;
    if (A->dtype != MR_F32 && A->dtype != MR_F16 && A->dtype != MR_BF16) return MR_ERR_UNSUPPORTED;
    if (A->n_rows > 0 && (!y || (A->nnz > 0 && (!x || !A->colidx || !A->vals)))) return MR_ERR_INVALID_ARG;
    const long long items = (long long)A->n_rows + A->nnz;
    if (items > kNoAllocMaxItems) {
        note_error("mr_spmv_merbit_noalloc: n_rows + nnz exceeds the 2^24 merge items of the static scratch");
        return MR_ERR_UNSUPPORTED;
    }
    if (A->n_rows == 0) return MR_OK;
    void* base = nullptr;
    MR_TRY(scratch_address(&base));
    unsigned char* b = static_cast<unsigned char*>(base);
    MerbitPlan p;
    p.sigma = kNoAllocSigma;
    p.block = 1024;  // persistent kernel
    p.n_rows = A->n_rows;
    p.nnz = A->nnz;
    p.lane_num = (int)((items + kNoAllocSigma - 1) / kNoAllocSigma);
    p.tile_num = (p.lane_num + 31) / 32;
    p.tile_x = reinterpret_cast<uint32_t*>(b + kOffTileX);
    p.tile_y = reinterpret_cast<uint32_t*>(b + kOffTileY);
    p.lane_desc = b + kOffDesc;
    p.carry = reinterpret_cast<float*>(b + kOffCarry);
    p.ticket = reinterpret_cast<int*>(b + kOffTicket);
    cudaStream_t st = as_stream(stream);
    // the matrix check, as at plan creation: its flag lives in the array and
    // its answer comes back through a host word (no allocation either side)
    int* flag = reinterpret_cast<int*>(b + kOffFlag);
    MR_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
    MR_TRY(validate_csr_async(*A, flag, st));
    int bad = 0;
    MR_CUDA_TRY(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    MR_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) {
        note_error("mr_spmv_merbit_noalloc: malformed CSR (rowptr or a column index out of range)");
        return MR_ERR_INVALID_ARG;
    }
    MR_CUDA_TRY(cudaMemsetAsync(p.ticket, 0, sizeof(int), st));
    MR_TRY(launch_merbit_plan(A->rowptr, A->n_rows, (int)A->nnz, p.sigma, p.lane_num, p.tile_num, p.tile_x, p.tile_y,
                              p.lane_desc, st));
    return launch_merbit_spmv(p, A->colidx, A->vals, A->dtype, x, y, p.carry, st);
}
