// Storage element types of the shear-warp kernels (float32, or bfloat16 read
// into FP32 arithmetic), the scalar column-pair FMA they issue, and the
// asynchronous-copy helpers beyond tma.cuh's tensor loads.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tma.cuh"

namespace petl {
namespace shear {

__device__ __forceinline__ float2 dup(float a) { return make_float2(a, a); }

// kAlign is the TMA x-coordinate granule (16 bytes) in elements.
template <class T>
struct Store;
template <>
struct Store<float> {
    static constexpr int kAlign = 4;
    static __device__ __forceinline__ float ld(float x) { return x; }
    static __device__ __forceinline__ float st(float x) { return x; }
    static __device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
    static __device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
};
template <>
struct Store<__nv_bfloat16> {
    static constexpr int kAlign = 8;
    static __device__ __forceinline__ float ld(__nv_bfloat16 x) { return __bfloat162float(x); }
    static __device__ __forceinline__ __nv_bfloat16 st(float x) { return __float2bfloat16_rn(x); }
    static __device__ __forceinline__ float2 ld2(const __nv_bfloat16* p)
    {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    }
    static __device__ __forceinline__ void st2(__nv_bfloat16* p, float2 v)
    {
        *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
    }
};

// Two scalar FMAs on a column pair.  Scalar FFMA issues at the full FP32
// rate with two warps per scheduler; the packed f32x2 form needs about four
// times the warps to reach the same rate on this part.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
}

}  // namespace shear

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Plain bulk copy global -> this CTA's shared memory (no tensor map, no
// multicast): both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace petl
