// Internal helpers shared by the libmr CUDA sources (sm_100a only).
#ifndef MR_COMMON_CUH
#define MR_COMMON_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mr.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libmr is written for sm_100a (B200) only"
#endif

namespace mr {

// Records a CUDA failure in the calling thread's last-error slot.
void note_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void note_error(const char* msg);

#define MR_CUDA_TRY(expr)                                                   \
    do {                                                                    \
        cudaError_t mr_e_ = (expr);                                         \
        if (mr_e_ != cudaSuccess) {                                         \
            ::mr::note_cuda_error(mr_e_, #expr, __FILE__, __LINE__);        \
            return MR_ERR_CUDA;                                             \
        }                                                                   \
    } while (0)

#define MR_TRY(expr)                  \
    do {                              \
        int mr_s_ = (expr);           \
        if (mr_s_ != MR_OK) return mr_s_; \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int sm_count()
{
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached = n > 0 ? n : 148;
    }
    return cached;
}

inline size_t dtype_size(int dt) { return dt == MR_F32 ? 4 : 2; }

// ---- value types: FP32 / FP16 / BF16 storage, FP32 arithmetic ----------
template <typename V> struct ValueTraits;
template <> struct ValueTraits<float> {
    static __device__ __forceinline__ float f(float v) { return v; }
};
template <> struct ValueTraits<__half> {
    static __device__ __forceinline__ float f(__half v) { return __half2float(v); }
};
template <> struct ValueTraits<__nv_bfloat16> {
    static __device__ __forceinline__ float f(__nv_bfloat16 v) { return __bfloat162float(v); }
};

// Four consecutive values as one vector load (16 B for FP32, 8 B for 16-bit).
template <typename V> struct Vec4;
template <> struct Vec4<float> {
    using T = float4;
    static __device__ __forceinline__ void unpack(const T& t, float (&o)[4]) { o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w; }
};
template <> struct Vec4<__half> {
    using T = uint2;
    static __device__ __forceinline__ void unpack(const T& t, float (&o)[4])
    {
        __half2 a = *reinterpret_cast<const __half2*>(&t.x);
        __half2 b = *reinterpret_cast<const __half2*>(&t.y);
        float2 fa = __half22float2(a), fb = __half22float2(b);
        o[0] = fa.x; o[1] = fa.y; o[2] = fb.x; o[3] = fb.y;
    }
};
template <> struct Vec4<__nv_bfloat16> {
    using T = uint2;
    static __device__ __forceinline__ void unpack(const T& t, float (&o)[4])
    {
        __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&t.x);
        __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&t.y);
        float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
        o[0] = fa.x; o[1] = fa.y; o[2] = fb.x; o[3] = fb.y;
    }
};

// ---- cache-hinted loads ---------------------------------------------------
// Matrix streams (colidx / values / descriptors) are read once per SpMV:
// load them evict-first so they do not push x out of L2.
__device__ __forceinline__ int4 ld_stream(const int4* p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ unsigned ld_stream(const unsigned* p) { return __ldcs(p); }
__device__ __forceinline__ unsigned long long ld_stream(const unsigned long long* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ld_stream(const uint2* p) { return __ldcs(p); }
__device__ __forceinline__ __half ld_stream(const __half* p)
{
    unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
    return __ushort_as_half(u);
}
__device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16* p)
{
    unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
    return __ushort_as_bfloat16(u);
}

// Streams that the persistent SpMV reads once: bypass L1 (so L1 holds only
// x) and mark them evict-first in L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ int4 ld_na(const int4* p, uint64_t pol)
{
    int4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_na(const float4* p, uint64_t pol)
{
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ uint2 ld_na(const uint2* p, uint64_t pol)
{
    uint2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ unsigned ld_na(const unsigned* p, uint64_t pol)
{
    unsigned v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ unsigned long long ld_na(const unsigned long long* p, uint64_t pol)
{
    unsigned long long v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
    return v;
}

// x is gathered many times per SpMV: keep it in L2 (evict-last policy) and
// use the read-only path.
__device__ __forceinline__ uint64_t l2_evict_last_policy()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_x(const float* p, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

__host__ __device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

// x gather variants: 0 = read-only path, allocate in L1; 1 = read-only
// path without L1 allocation; 2 = L2 only (.cg). All keep the line in L2.
__device__ __forceinline__ float ld_x_mode(const float* p, uint64_t pol, int mode)
{
    float v;
    if (mode == 1)
        asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    else if (mode == 2)
        asm("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    else
        asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

// ---- warp helpers ----------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace mr

#endif
