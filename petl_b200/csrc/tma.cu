// Host side of the TMA helpers: tensor-map encoding through the driver entry
// point, and the device error word that bounded waits report into.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "common.cuh"
#include "tma.cuh"

namespace petl {

namespace {
__device__ int g_device_error = 0;

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn()
{
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}
}  // namespace

namespace {
std::atomic<int> g_force_timeout{0};
}

unsigned wait_limit() { return g_force_timeout.load(std::memory_order_relaxed) ? 0u : kWaitLimit; }

int* device_error_ptr()
{
    static std::mutex mu;
    static int* ptr[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
        ptr[dev] = static_cast<int*>(p);
    }
    return ptr[dev];
}

bool encode_tensor_map(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, int elem_bytes)
{
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    if (elem_bytes != 4 && elem_bytes != 2) return false;
    if (reinterpret_cast<uintptr_t>(base) & 15) return false;
    for (int i = 0; i + 1 < rank; i++)
        if (strides_bytes[i] & 15) return false;
    if ((box[0] * uint32_t(elem_bytes)) & 15) return false;
    cuuint64_t d[5], s[4];
    cuuint32_t b[5], e[5];
    for (int i = 0; i < rank; i++) {
        d[i] = dims[i];
        b[i] = box[i];
        e[i] = 1;
        if (b[i] == 0 || b[i] > 256) return false;
    }
    for (int i = 0; i + 1 < rank; i++) s[i] = strides_bytes[i];
    const CUtensorMapDataType dt = elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const CUresult r = fn(map, dt, cuuint32_t(rank), const_cast<void*>(base), d, s, b, e,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace petl

extern "C" int petl_device_error_flag(void)
{
    int* p = petl::device_error_ptr();
    if (!p) return -1;
    int h = 0;
    if (cudaMemcpy(&h, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (h) {
        const int z = 0;
        cudaMemcpy(p, &z, sizeof(int), cudaMemcpyHostToDevice);
    }
    return h;
}

extern "C" int petl_force_wait_timeout(int on)
{
    petl::g_force_timeout.store(on ? 1 : 0, std::memory_order_relaxed);
    return 0;
}
