// Internal declarations shared between the libmr sources.
#ifndef MR_INTERNAL_HPP
#define MR_INTERNAL_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "mr.h"

namespace mr {

// MERBIT plan: the reference's descriptor arrays plus the carry scratch.
struct MerbitPlan {
    int sigma = 14;
    int block = 256;
    int n_rows = 0;
    int64_t nnz = 0;
    int lane_num = 0;
    int tile_num = 0;
    uint32_t* tile_x = nullptr;   // tile_num + 1
    uint32_t* tile_y = nullptr;   // tile_num + 1
    void* lane_desc = nullptr;    // lane_num words (4 or 8 bytes)
    float* carry = nullptr;       // tile_num carries
    int* ticket = nullptr;        // persistent kernel's completion counter (starts at 0)
    // hub cache (persistent kernel only): the most-used columns' x values are
    // staged in shared memory; colh is the plan's copy of colidx with hub
    // columns replaced by (0x80000000 | slot); hub_cols[slot] = column
    int32_t* colh = nullptr;
    int32_t* hub_cols = nullptr;
    int hub_k = 0;
    double hub_coverage = 0.0;    // share of nonzeros whose column is a hub
    int hub_limit = 0;            // cap on hub slots (0: as many as fit)
    int gather_mode = 0;          // x gather cache path (ld_x_mode)
    int device = 0;
    // persistent kernel: tile chunk of each CTA, chunk_start[c] .. chunk_start[c+1],
    // balanced by estimated cost (chunks + 1 entries); nullptr: equal tile counts
    int32_t* chunk_start = nullptr;
    int chunks = 0;
    // the carry run that crosses the start of chunk c, c = 1 .. chunks - 1:
    // {row, first tile, last tile, kind}; kind 0: none finishes in chunk c,
    // 1: all its tiles lie in chunks c - 1 and c (finished by whichever of
    // the two CTAs ends second), 2: it starts earlier (finished by the last
    // CTA). chunks + 1 entries; boundary_flag: chunks + 1 arrival counters
    int4* boundary_run = nullptr;
    int* boundary_flag = nullptr;
};

int launch_merbit_plan(const int* rowptr, int nrow, int nnz, int sigma, int lane_num, int tile_num, uint32_t* tile_x,
                       uint32_t* tile_y, void* lane_desc, cudaStream_t st);
int launch_merbit_spmv(const MerbitPlan& p, const int* colidx, const void* vals, int dtype, const float* x, float* y,
                       float* carry, cudaStream_t st);
bool merbit_sigma_supported(int sigma);
// builds the hub cache of a persistent-kernel plan (no-op when it would not pay)
int build_hub_cache(MerbitPlan& p, const mr_csr_view& A, cudaStream_t st);
// cost-balanced CTA chunks of a persistent-kernel plan (after the hub cache)
int build_chunk_bounds(MerbitPlan& p, const int* colidx, cudaStream_t st);
// frees every device buffer a plan owns
void free_plan_buffers(MerbitPlan& p);
// CTAs of the persistent kernel for a plan of tile_num tiles on this device
int persistent_grid(int tile_num);
// largest number of hub slots that fit beside the SIGMA staging buffers
int hub_capacity(int sigma);

int launch_csr_spmv(int n, int64_t nnz, const int* rowptr, const int* colidx, const void* vals, int dtype,
                    const float* x, float* y, cudaStream_t st);

// batched SpMV internals (operand tables built by the caller)
size_t batch_op_bytes(int dtype, int sigma);
int batch_fill_op(void* dst, int dtype, int sigma, const MerbitPlan& p, const mr_csr_view& A, const float* x, float* y,
                  float* carry);
int batch_launch_ops(int dtype, int sigma, const void* d_ops, const long long* d_prefix, int count,
                     long long total_tiles, cudaStream_t st);

// permutation
int permute_csr(const mr_csr_view& A, const int32_t* perm, int32_t* out_rowptr, int32_t* out_colidx, void* out_vals,
                cudaStream_t st);
int launch_permute_vector(int n, const int32_t* perm, const float* in, float* out, int inverse, cudaStream_t st);
int launch_perm_invert(int n, const int32_t* perm, int32_t* inv, int* bad_flag, cudaStream_t st);
int check_perm(const int32_t* perm, int n, int* valid, cudaStream_t st);
int validate_csr(const mr_csr_view& A, int* ok, cudaStream_t st);
// enqueues the checks of validate_csr; *bad_dev (zeroed by the caller) gets
// 1 for a malformed rowptr, 2 for a column index outside [0, n_cols)
int validate_csr_async(const mr_csr_view& A, int* bad_dev, cudaStream_t st);

// device scan: out[i] = sum_{j<i} in[j], out[n] = total (n + 1 outputs)
int exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t st);
size_t scan_workspace_bytes(int64_t n);
int exclusive_scan_i32_ws(const int32_t* in, int32_t* out, int64_t n, void* ws, cudaStream_t st);

// reuse distance
int rd_hist_exact(const int32_t* stream, int64_t nnz, int32_t ncols, int32_t sector, const int32_t* edges,
                  int32_t nedges, int64_t* counts, int64_t* valid, cudaStream_t st);
int rd_hist_sampled(const int32_t* stream, int32_t nnz, int32_t samples, int32_t sector, int32_t rd_cap, int32_t hll_p,
                    int32_t max_scan, uint32_t seed, const int32_t* edges, int32_t nedges, int64_t* counts,
                    int64_t* stats, float* est, int32_t* status, int32_t* pos, cudaStream_t st);

// host-side pGOrder
int pgorder_host(int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t vsize, int32_t width,
                 int32_t threads, uint32_t* perm_new2old);
int32_t pgorder_width(int32_t n, int64_t nnz);

// stream-ordered scratch
// pGOrder on the device (one warp per block of ids), bit-identical to
// pgorder_host; MR_ERR_UNSUPPORTED when the block or key range does not fit
// its 16-bit shared-memory queue.
int pgorder_gpu(int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t nnz, int32_t vsize, int32_t width,
                uint32_t* perm, cudaStream_t st);

// Stable LSD radix sort of (key, value) pairs over the low `bits` bits of the
// keys, 8 bits per pass, ping-ponging with kbuf / vbuf: on return keys / vals
// point at the buffers that hold the sorted pairs.
int radix_sort_pairs_u32(uint32_t*& keys, int32_t*& vals, uint32_t* kbuf, int32_t* vbuf, int64_t n, int bits,
                         cudaStream_t st);

// Runs a set-up step (kernel attributes and the like) once per device: the
// first call on each device runs it with that device current and keeps its
// status; later calls on the device return the kept status.
struct PerDeviceOnce {
    std::mutex mu;
    uint64_t done = 0;
    cudaError_t status[64] = {};
    template <typename F> cudaError_t run(F&& f)
    {
        int dev = 0;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return f();  // beyond the table: every call
        std::lock_guard<std::mutex> lk(mu);
        if (!((done >> dev) & 1u)) {
            status[dev] = f();
            done |= 1ull << dev;
        }
        return status[dev];
    }
};

// Stream-ordered pool of the current device for temporaries (DevBuf). It
// keeps freed memory for reuse instead of returning it at every
// synchronisation (the default pool's behaviour), so repeated calls do not
// map their scratch again; mr_release_scratch() trims it.
cudaMemPool_t scratch_pool();

struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf()
    {
        if (p) cudaFreeAsync(p, st);
    }
    int alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        if (bytes == 0) bytes = 16;
        cudaMemPool_t pool = scratch_pool();
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, s) : cudaMallocAsync(&p, bytes, s);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return MR_ERR_NOMEM;
        }
        return MR_OK;
    }
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

}  // namespace mr

// opaque handle of include/mr.h
struct mr_merbit_plan {
    mr::MerbitPlan p;
};

#endif
