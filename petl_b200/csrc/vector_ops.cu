// Elementwise MLEM/OSEM glue and FP64 reductions on the device.
//
// The elementwise rules are the reference dataCube rules
// (src/data_cube.cpp:97-166): DIV gives 0 where the divisor is 0, RDIV gives
// 0 where the denominator is 0, RECIPROCAL gives a caller value at 0.  The
// reference runs them as OpenMP loops on the host between GPU calls; here
// they are fused, grid-strided, 128-bit vectorised kernels so the iteration
// stays on the device.  Reductions accumulate in double (the reference's CPU
// inner products accumulate in double, src/data_cube.cpp:320-440) with a
// deterministic two-pass block reduction.
#include <mutex>

#include "common.cuh"
#include "reduce.cuh"

namespace petl {

namespace {

template <class Op>
__global__ void k_map2(float* __restrict__ x, const float* __restrict__ y, long long n, Op op)
{
    const long long n4 = n >> 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    float4* x4 = reinterpret_cast<float4*>(x);
    const float4* y4 = reinterpret_cast<const float4*>(y);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 a = x4[i];
        const float4 b = y4[i];
        a.x = op(a.x, b.x);
        a.y = op(a.y, b.y);
        a.z = op(a.z, b.z);
        a.w = op(a.w, b.w);
        x4[i] = a;
    }
    for (long long i = (n4 << 2) + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = op(x[i], y[i]);
}

struct OpMul { __device__ float operator()(float a, float b) const { return a * b; } };
struct OpDiv { __device__ float operator()(float a, float b) const { return b == 0.0f ? 0.0f : a / b; } };
// out = num / denom with denom stored in the first operand
struct OpRDiv { __device__ float operator()(float den, float num) const { return den == 0.0f ? 0.0f : num / den; } };
// d/d(Pf) of the Poisson negative log-likelihood sum(Pf - g log Pf) over
// Pf > 0 (the bins the log-likelihood sums), Pf stored in the first operand
struct OpPoissonGrad {
    __device__ float operator()(float pf, float g) const { return pf > 0.0f ? 1.0f - g / pf : 0.0f; }
};

__global__ void k_reciprocal(float* __restrict__ x, long long n, float v)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = x[i] == 0.0f ? v : 1.0f / x[i];
}

__global__ void k_axpby(float* __restrict__ x, const float* __restrict__ y, float a, float b, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = a * x[i] + b * y[i];
}

__global__ void k_mlem_update(float* __restrict__ f, const float* __restrict__ d, const float* __restrict__ s,
                              long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float den = s[i];
        f[i] *= den == 0.0f ? 0.0f : d[i] / den;
    }
}

__global__ void k_osl_update(float* __restrict__ f, const float* __restrict__ d, const float* __restrict__ s,
                             const float* __restrict__ Df, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float sv = s[i];
        const float den = fmaxf(0.1f * sv, Df[i] + sv);
        f[i] *= den == 0.0f ? 0.0f : d[i] / den;
    }
}

struct DotTerm {
    const float *x, *y, *w;
    __device__ double operator()(long long i) const
    {
        const double p = double(x[i]) * double(y[i]);
        return w ? p * double(w[i]) : p;
    }
};

struct LoglikTerm {
    const float *g, *pf;
    __device__ double operator()(long long i) const
    {
        const float p = pf[i];
        return p > 0.0f ? double(g[i]) * log(double(p)) - double(p) : 0.0;
    }
};

int grid_for(long long n, int block)
{
    const long long want = (n + block - 1) / block;
    const long long cap = (long long)sm_count() * 8;
    return int(want < cap ? (want < 1 ? 1 : want) : cap);
}

template <class Op>
__global__ void k_map2_scalar(float* __restrict__ x, const float* __restrict__ y, long long n, Op op)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = op(x[i], y[i]);
}

template <class Op>
int map2(float* x, const float* y, long long n, void* stream, const char* name)
{
    PETL_REQUIRE(x && y && n >= 0, std::string(name) + ": invalid arguments");
    if (n == 0) return 0;
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    if (aligned)
        k_map2<<<grid_for(n / 4 + 1, 256), 256, 0, as_stream(stream)>>>(x, y, n, Op());
    else
        k_map2_scalar<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(x, y, n, Op());
    PETL_LAUNCH_CHECK(name);
    return 0;
}

}  // namespace

}  // namespace petl

using namespace petl;

extern "C" {

int petl_multiply_dev(float* x, const float* y, long long n, void* stream)
{
    return map2<OpMul>(x, y, n, stream, "multiply");
}

int petl_divide_dev(float* x, const float* y, long long n, void* stream)
{
    return map2<OpDiv>(x, y, n, stream, "divide");
}

int petl_rdivide_dev(const float* num, float* denom, long long n, void* stream)
{
    return map2<OpRDiv>(denom, num, n, stream, "rdivide");
}

int petl_poisson_grad_dev(float* Pf, const float* g, long long n, void* stream)
{
    return map2<OpPoissonGrad>(Pf, g, n, stream, "poisson_grad");
}

int petl_reciprocal_dev(float* x, long long n, float v, void* stream)
{
    PETL_REQUIRE(x && n >= 0, "reciprocal: invalid arguments");
    if (n == 0) return 0;
    k_reciprocal<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(x, n, v);
    PETL_LAUNCH_CHECK("reciprocal");
    return 0;
}

int petl_axpby_dev(float* x, const float* y, float a, float b, long long n, void* stream)
{
    PETL_REQUIRE(x && y && n >= 0, "axpby: invalid arguments");
    if (n == 0) return 0;
    k_axpby<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(x, y, a, b, n);
    PETL_LAUNCH_CHECK("axpby");
    return 0;
}

int petl_mlem_update_dev(float* f, const float* d, const float* sens, long long n, void* stream)
{
    PETL_REQUIRE(f && d && sens && n >= 0, "mlem_update: invalid arguments");
    if (n == 0) return 0;
    k_mlem_update<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(f, d, sens, n);
    PETL_LAUNCH_CHECK("mlem_update");
    return 0;
}

int petl_osl_update_dev(float* f, const float* d, const float* sens, const float* Df, long long n, void* stream)
{
    PETL_REQUIRE(f && d && sens && Df && n >= 0, "osl_update: invalid arguments");
    if (n == 0) return 0;
    k_osl_update<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(f, d, sens, Df, n);
    PETL_LAUNCH_CHECK("osl_update");
    return 0;
}

int petl_dot_dev(const float* x, const float* y, const float* w, long long n, double* out, void* stream)
{
    PETL_REQUIRE(x && y && out && n >= 0, "dot: invalid arguments");
    return reduce_sum(DotTerm{x, y, w}, n, out, as_stream(stream), "dot");
}

int petl_loglik_dev(const float* g, const float* Pf, long long n, double* out, void* stream)
{
    PETL_REQUIRE(g && Pf && out && n >= 0, "loglik: invalid arguments");
    return reduce_sum(LoglikTerm{g, Pf}, n, out, as_stream(stream), "loglik");
}

}  // extern "C"
