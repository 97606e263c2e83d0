// Shared internals of libpetl.so: error reporting, stream casts, launch
// checks and rounding-pinned float helpers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/petl_device.h"

namespace petl {

// Records an error message for the calling thread (read by petl_last_error).
void set_error(const std::string& msg);
void clear_error();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Checks a CUDA call; on failure records the message and returns its code.
#define PETL_CUDA(expr)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            ::petl::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));       \
            return int(e_);                                                              \
        }                                                                                \
    } while (0)

// Counts kernel launches issued by the library (petl_launch_count()).
void note_launch();

// Checks the launch that was just issued (and counts it).
#define PETL_LAUNCH_CHECK(name)                                                          \
    do {                                                                                 \
        ::petl::note_launch();                                                           \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) {                                                         \
            ::petl::set_error(std::string(name) + " launch: " + cudaGetErrorString(e_)); \
            return int(e_);                                                              \
        }                                                                                \
    } while (0)

#define PETL_REQUIRE(cond, msg)                 \
    do {                                        \
        if (!(cond)) {                          \
            ::petl::set_error(msg);             \
            return -1;                          \
        }                                       \
    } while (0)

inline unsigned ceil_div(long long a, long long b) { return unsigned((a + b - 1) / b); }

// Number of SMs on the current device (cached per device).
int sm_count();

// Stream-ordered scratch from the library's own memory pool on the current
// device, which keeps freed blocks for reuse (free with cudaFreeAsync).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st);

// Geometry sanity check shared by the entry points.
bool geom_valid(const petl_geom* G, std::string* why);

// ---------------------------------------------------------------------------
// Rounding-pinned arithmetic.  The footprint weights of the forward projector
// and of its exact adjoint are evaluated by the same helper functions; the
// _rn intrinsics stop the compiler from contracting them differently in the
// two kernels, so both see bit-identical weights.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// overlap of the bin [i-1/2, i+1/2] with the interval [c-w, c+w] (index units)
__device__ __forceinline__ float box_overlap(int i, float c, float w)
{
    const float lo = fmaxf(fsub(float(i), 0.5f), fsub(c, w));
    const float hi = fminf(fadd(float(i), 0.5f), fadd(c, w));
    return fsub(hi, lo);
}

}  // namespace petl
