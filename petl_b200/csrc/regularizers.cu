// Relative-difference and p-Huber total-variation penalties on a 3-D array
// [N1][N2][N3] (N3 fastest), 26- (or 6-) neighbour stencils with clamped
// borders.
//
// Restates src/relative_differences.cu:13-173 (RD potential, its derivative,
// clip of f < 1e-8 to zero before the gradient) and src/total_variation.cu:
// 21-78 (Huber with USE_P_HUBER), 80-572 (cost / quadratic form / gradient
// terms, including the planar N1 == 1 case) and 574-811 (host parameter
// conventions: beta <= 0 -> 1, delta < 1e-8 -> 1e-8).  Differences from the
// reference: the thread mapping puts the fastest thread index on the fastest
// array index (the reference maps threadIdx.x to the slowest axis), sums are
// accumulated in double, and pow() is the accurate libdevice powf rather
// than the fast-math approximation.
#include <cmath>
#include "common.cuh"
#include "reduce.cuh"

namespace petl {

namespace {

struct Dims {
    int n1, n2, n3;
};

__device__ __forceinline__ size_t vidx(const Dims& d, int i, int j, int k)
{
    return (size_t(i) * d.n2 + j) * d.n3 + k;
}

// --- relative differences (src/relative_differences.cu:13-28) -------------
__device__ __forceinline__ float rd_clip(float v) { return v < 0.00000001f ? 0.0f : v; }

__device__ __forceinline__ float rd_pot(float x, float y, float delta)
{
    if (x == y) return 0.0f;
    const float d = x - y;
    return d * d / ((x + y) + delta * fabsf(d));
}

__device__ __forceinline__ float rd_dpot(float x, float y, float delta)
{
    if (x == 0.0f && y == 0.0f) return 0.0f;
    const float d = x - y;
    const float s = x + y + delta * fabsf(d);
    return d * (delta * fabsf(d) + x + 3.0f * y) / (s * s);
}

// --- p-Huber (src/total_variation.cu:33-78) --------------------------------
struct HuberP {
    float p, delta, slope, shift;
    __device__ __forceinline__ float h(float x) const
    {
        const float a = fabsf(x);
        return a <= delta ? 0.5f * x * x : slope * powf(a, p) + shift;
    }
    __device__ __forceinline__ float dh(float x) const
    {
        const float a = fabsf(x);
        return a <= delta ? x : p * slope * powf(a, p) / x;
    }
    __device__ __forceinline__ float ddh(float x) const
    {
        const float a = fabsf(x);
        return a <= delta ? 1.0f : p * slope * powf(a, p - 2.0f);
    }
};

HuberP make_huber(float& delta, float& beta, float p)
{
    // anisotropicTotalVariation_* argument handling + setConstantMemoryParameters
    if (beta <= 0.0) beta = 1.0;
    if (delta < 1.0e-8) delta = float(1.0e-8);
    HuberP h;
    h.p = p;
    h.delta = delta;
    h.slope = float(std::pow(double(delta), 2.0 - p) / p);
    h.shift = float(double(delta) * delta * (0.5 - 1.0 / p));
    return h;
}

// Visits the neighbour classes of the stencil: F(di,dj,dk,cls) with cls
// 1 = face, 2 = edge, 3 = corner.  planar: only j/k neighbours (N1 == 1).
template <class F>
__device__ __forceinline__ void for_neighbours(bool planar, int numNeighbors, F fn)
{
#pragma unroll
    for (int di = -1; di <= 1; di++)
#pragma unroll
        for (int dj = -1; dj <= 1; dj++)
#pragma unroll
            for (int dk = -1; dk <= 1; dk++) {
                const int cls = (di != 0) + (dj != 0) + (dk != 0);
                if (cls == 0) continue;
                if (planar && di != 0) continue;
                if (numNeighbors == 6 && cls > 1) continue;
                fn(di, dj, dk, cls);
            }
}

__device__ __forceinline__ float combine(float s1, float s2, float s3, float beta)
{
    const float d1 = 1.0f * beta, d2 = 0.7071067811865475f * beta, d3 = 0.5773502691896258f * beta;
    return s1 * d1 + s2 * d2 + s3 * d3;
}

__global__ void __launch_bounds__(256)
k_rd_gradient(const float* __restrict__ f, float* __restrict__ Df, Dims d, float delta, float beta)
{
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.n3 || j >= d.n2) return;
    const float x = rd_clip(__ldg(&f[vidx(d, i, j, k)]));
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for_neighbours(false, 26, [&](int di, int dj, int dk, int cls) {
        const int ii = min(d.n1 - 1, max(0, i + di)), jj = min(d.n2 - 1, max(0, j + dj)),
                  kk = min(d.n3 - 1, max(0, k + dk));
        s[cls] += rd_dpot(x, rd_clip(__ldg(&f[vidx(d, ii, jj, kk)])), delta);
    });
    Df[vidx(d, i, j, k)] = combine(s[1], s[2], s[3], beta);
}

struct RdCostTerm {
    const float* f;
    Dims d;
    float delta, beta;
    __device__ double operator()(long long idx) const
    {
        const int k = int(idx % d.n3), j = int((idx / d.n3) % d.n2), i = int(idx / ((long long)d.n3 * d.n2));
        const float x = rd_clip(f[idx]);
        double s[4] = {0, 0, 0, 0};
        for_neighbours(false, 26, [&](int di, int dj, int dk, int cls) {
            const int ii = min(d.n1 - 1, max(0, i + di)), jj = min(d.n2 - 1, max(0, j + dj)),
                      kk = min(d.n3 - 1, max(0, k + dk));
            s[cls] += rd_pot(x, rd_clip(f[vidx(d, ii, jj, kk)]), delta);
        });
        return s[1] * double(1.0f * beta) + s[2] * double(0.7071067811865475f * beta) +
               s[3] * double(0.5773502691896258f * beta);
    }
};

__global__ void __launch_bounds__(256)
k_tv_gradient(const float* __restrict__ f, float* __restrict__ Df, Dims d, HuberP hb, float beta, int nbrs)
{
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.n3 || j >= d.n2) return;
    const bool planar = d.n1 == 1;
    const float x = __ldg(&f[vidx(d, i, j, k)]);
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for_neighbours(planar, nbrs, [&](int di, int dj, int dk, int cls) {
        const int ii = min(d.n1 - 1, max(0, i + di)), jj = min(d.n2 - 1, max(0, j + dj)),
                  kk = min(d.n3 - 1, max(0, k + dk));
        s[cls] += hb.dh(x - __ldg(&f[vidx(d, ii, jj, kk)]));
    });
    Df[vidx(d, i, j, k)] = combine(s[1], s[2], s[3], beta);
}

struct TvCostTerm {
    const float* f;
    Dims d;
    HuberP hb;
    float beta;
    int nbrs;
    __device__ double operator()(long long idx) const
    {
        const int k = int(idx % d.n3), j = int((idx / d.n3) % d.n2), i = int(idx / ((long long)d.n3 * d.n2));
        const float x = f[idx];
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        for_neighbours(d.n1 == 1, nbrs, [&](int di, int dj, int dk, int cls) {
            const int ii = min(d.n1 - 1, max(0, i + di)), jj = min(d.n2 - 1, max(0, j + dj)),
                      kk = min(d.n3 - 1, max(0, k + dk));
            s[cls] += hb.h(x - f[vidx(d, ii, jj, kk)]);
        });
        return double(combine(s[1], s[2], s[3], beta));
    }
};

struct TvQuadTerm {
    const float *f, *dd;
    Dims d;
    HuberP hb;
    float beta;
    int nbrs;
    __device__ double operator()(long long idx) const
    {
        const int k = int(idx % d.n3), j = int((idx / d.n3) % d.n2), i = int(idx / ((long long)d.n3 * d.n2));
        const float x = f[idx], xd = dd[idx];
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        for_neighbours(d.n1 == 1, nbrs, [&](int di, int dj, int dk, int cls) {
            const int ii = min(d.n1 - 1, max(0, i + di)), jj = min(d.n2 - 1, max(0, j + dj)),
                      kk = min(d.n3 - 1, max(0, k + dk));
            const size_t q = vidx(d, ii, jj, kk);
            const float e = xd - dd[q];
            s[cls] += hb.ddh(x - f[q]) * e * e;
        });
        return double(combine(s[1], s[2], s[3], beta));
    }
};

bool dims_ok(int n1, int n2, int n3) { return n1 > 0 && n2 > 0 && n3 > 0 && n1 <= 65535; }

}  // namespace
}  // namespace petl

using namespace petl;

extern "C" {

int petl_rd_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, void* stream)
{
    PETL_REQUIRE(f && Df && dims_ok(N1, N2, N3), "rd_gradient: invalid arguments");
    const Dims d{N1, N2, N3};
    dim3 block(32, 8, 1), grid(ceil_div(N3, 32), ceil_div(N2, 8), unsigned(N1));
    k_rd_gradient<<<grid, block, 0, as_stream(stream)>>>(f, Df, d, delta, beta);
    PETL_LAUNCH_CHECK("rd_gradient");
    return 0;
}

int petl_rd_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, double* out, void* stream)
{
    PETL_REQUIRE(f && out && dims_ok(N1, N2, N3), "rd_cost: invalid arguments");
    const Dims d{N1, N2, N3};
    return reduce_sum(RdCostTerm{f, d, delta, beta}, (long long)N1 * N2 * N3, out, as_stream(stream), "rd_cost");
}

int petl_tv_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, void* stream)
{
    PETL_REQUIRE(f && Df && dims_ok(N1, N2, N3), "tv_gradient: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    dim3 block(32, 8, 1), grid(ceil_div(N3, 32), ceil_div(N2, 8), unsigned(N1));
    k_tv_gradient<<<grid, block, 0, as_stream(stream)>>>(f, Df, d, hb, beta, numNeighbors == 6 ? 6 : 26);
    PETL_LAUNCH_CHECK("tv_gradient");
    return 0;
}

int petl_tv_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, float p, int numNeighbors,
                     double* out, void* stream)
{
    PETL_REQUIRE(f && out && dims_ok(N1, N2, N3), "tv_cost: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    return reduce_sum(TvCostTerm{f, d, hb, beta, numNeighbors == 6 ? 6 : 26}, (long long)N1 * N2 * N3, out,
                      as_stream(stream), "tv_cost");
}

int petl_tv_quadform_dev(const float* f, const float* dvec, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, double* out, void* stream)
{
    PETL_REQUIRE(f && dvec && out && dims_ok(N1, N2, N3), "tv_quadform: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    return reduce_sum(TvQuadTerm{f, dvec, d, hb, beta, numNeighbors == 6 ? 6 : 26}, (long long)N1 * N2 * N3, out,
                      as_stream(stream), "tv_quadform");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Gaussian filter (src/relative_differences.cu:314-411, 753-800).  The
// reference weight exp(-(di^2+dj^2+dk^2)/(2 sigma)) is taken with the
// distance to the CLAMPED neighbour index, which factorises per axis, so the
// 3-D (or 2-D over j,k, or 1-D over i) filter runs as separable 1-D passes;
// the normalisation by the weight sum factorises the same way.
// ---------------------------------------------------------------------------
namespace petl {
namespace {
__global__ void __launch_bounds__(256)
k_gauss_axis(const float* __restrict__ in, float* __restrict__ out, int N1, int N2, int N3, int axis, int radius,
             float denom)
{
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= N3 || j >= N2) return;
    const int n = axis == 0 ? N1 : axis == 1 ? N2 : N3;
    const int c = axis == 0 ? i : axis == 1 ? j : k;
    const size_t stride = axis == 0 ? size_t(N2) * N3 : axis == 1 ? size_t(N3) : 1;
    const size_t base = (size_t(i) * N2 + j) * N3 + k - size_t(c) * stride;
    float val = 0.0f, sum = 0.0f;
    for (int d = -radius; d <= radius; d++) {
        const int s = max(0, min(c + d, n - 1));
        const float w = expf(-denom * float((c - s) * (c - s)));
        val += w * in[base + size_t(s) * stride];
        sum += w;
    }
    out[(size_t(i) * N2 + j) * N3 + k] = val / sum;
}
}  // namespace

int launch_gaussian(float* f, int N1, int N2, int N3, float FWHM, int numDims, cudaStream_t st)
{
    const float sigma = FWHM / (2.0f * std::sqrt(2.0f * std::log(2.0f)));
    const int radius = int(std::ceil(std::sqrt(2.0f * std::log(10.0f)) * sigma));
    const float denom = 1.0f / (2.0f * sigma);
    const size_t n = size_t(N1) * N2 * N3;
    float* tmp = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&tmp), sizeof(float) * n, st));
    dim3 block(32, 8, 1), grid(ceil_div(N3, 32), ceil_div(N2, 8), unsigned(N1));
    int axes[3], na = 0;
    if (numDims == 1) axes[na++] = 0;
    else if (numDims == 2) { axes[na++] = 1; axes[na++] = 2; }
    else { axes[na++] = 0; axes[na++] = 1; axes[na++] = 2; }
    cudaError_t e = cudaSuccess;
    for (int a = 0; a < na && e == cudaSuccess; a++) {
        k_gauss_axis<<<grid, block, 0, st>>>(f, tmp, N1, N2, N3, axes[a], radius, denom);
        e = cudaGetLastError();
        note_launch();
        if (e == cudaSuccess) e = cudaMemcpyAsync(f, tmp, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
    }
    cudaFreeAsync(tmp, st);
    if (e != cudaSuccess) {
        set_error(std::string("gaussian_filter: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}
}  // namespace petl
