// Tensor-memory-accelerator (TMA) loads and mbarrier waits for sm_100a.
//
// Loads are plain tiled cp.async.bulk.tensor copies into this CTA's shared
// memory (no cluster multicast).  Every wait on an mbarrier is bounded: after
// kWaitLimit polls it records an error in the library's device error word
// and gives up, so a lost completion cannot hang the GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace petl {

// Device error word (petl_device_error_flag() reads and clears it); kernels
// receive its device address as an argument (device_error_ptr()).
enum : int {
    kErrWaitTimeout = 1,  // a bounded wait gave up
    kErrLayout = 2,       // a host-side bound on a kernel's layout (shift spread, table size) did not hold
};
int* device_error_ptr();

constexpr unsigned kWaitLimit = 1u << 22;

// The bound a launch passes to its waits on staged data: kWaitLimit, or 0
// (give up before polling) while petl_force_wait_timeout(1) is in effect
// (host; read when a launch's arguments are built).  The waits that drain
// copies in flight after a give-up always use kWaitLimit.
unsigned wait_limit();

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Non-blocking test of the given phase parity.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the given phase parity; false (and the error word set) on
// timeout.  limit 0 gives up without polling; any other limit polls up to
// kWaitLimit times (a poll loop with a run-time bound measured 20 % slower
// in the projector kernels than this compile-time one).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, unsigned limit = kWaitLimit)
{
    if (limit != 0)
        for (unsigned i = 0; i < kWaitLimit; i++)
            if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, kErrWaitTimeout);
    return false;
}

// Bounded wait that also ends when *abort is nonzero: another warp of the
// CTA gave up a wait, and the copy awaited here may never be started.  The
// flag is read only after an unsuccessful poll.  false on either; the error
// word is set on a timeout only (the warp that gave up has set it).
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t* bar, uint32_t parity, int* err, const volatile int* abort)
{
    for (unsigned i = 0; i < kWaitLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
    }
    if (err) atomicOr(err, kErrWaitTimeout);
    return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Host: encode a tiled tensor map of float32 (elem_bytes 4) or bfloat16
// (elem_bytes 2) elements, dims/box fastest first.  Returns false when the
// driver entry point is unavailable or the layout is not TMA-compatible (base
// 16-byte aligned, strides and the box's inner extent multiples of 16 bytes).
bool encode_tensor_map(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, int elem_bytes = 4);

}  // namespace petl
