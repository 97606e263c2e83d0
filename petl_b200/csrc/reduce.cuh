// Deterministic FP64 sum of a per-element term: one pass of block partials
// into stream-ordered scratch, one single-block pass that adds the partials
// in a fixed order.  Used by the dot products, the Poisson log-likelihood and
// the regularizer costs.
#pragma once
#include "common.cuh"

namespace petl {

template <int BLOCK>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[BLOCK / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < BLOCK / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;  // valid in thread 0
}

template <class Term>
__global__ void __launch_bounds__(256) k_reduce_partial(Term term, long long n, double* __restrict__ partial)
{
    double s = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) s += term(i);
    s = block_sum<256>(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <int UNUSED = 0>
__global__ void __launch_bounds__(256) k_reduce_final(const double* __restrict__ partial, int nb,
                                                      double* __restrict__ out)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) s += partial[i];
    s = block_sum<256>(s);
    if (threadIdx.x == 0) *out = s;
}

// Sums term(i) for i in [0, n) into *out (a device double).
template <class Term>
int reduce_sum(Term term, long long n, double* out, cudaStream_t st, const char* name)
{
    const long long want = (n + 255) / 256;
    const int nb = int(want < 1 ? 1 : (want > 4LL * sm_count() ? 4LL * sm_count() : want));
    double* part = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&part), sizeof(double) * nb, st));
    k_reduce_partial<<<nb, 256, 0, st>>>(term, n, part);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        k_reduce_final<0><<<1, 256, 0, st>>>(part, nb, out);
        note_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(part, st);
    if (e != cudaSuccess) {
        set_error(std::string(name) + ": " + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl
