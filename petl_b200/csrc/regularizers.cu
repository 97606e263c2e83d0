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

// the division as the reference's --use_fast_math build computes it (as in
// the gradient below)
__device__ __forceinline__ float rd_pot(float x, float y, float delta)
{
    if (x == y) return 0.0f;
    const float d = x - y;
    return __fdividef(d * d, (x + y) + delta * fabsf(d));
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

__device__ __forceinline__ float combine(float s1, float s2, float s3, float beta)
{
    const float d1 = 1.0f * beta, d2 = 0.7071067811865475f * beta, d3 = 0.5773502691896258f * beta;
    return s1 * d1 + s2 * d2 + s3 * d3;
}

// ---------------------------------------------------------------------------
// Gradient stencils, tiled: a CTA owns a 8 x 32 (j, k) column tile over a run
// of SPLANES planes i and marches along i with three halo planes (clamped
// indices, as the reference clamps its neighbours) in shared memory, so each
// voxel is read from global memory once per plane pass instead of 27 times
// with 27 index clamps.  The neighbour terms are summed per class in the
// order of for_neighbours.
// ---------------------------------------------------------------------------
constexpr int STJ = 8, STK = 32, SPLANES = 16;
constexpr int SHJ = STJ + 2, SHK = STK + 2;  // halo tile

// RD: the reference clips f < 1e-8 to zero before the gradient; the
// division is the fast approximate one (the reference builds with
// --use_fast_math).
struct RdGradOp {
    float delta;
    __device__ __forceinline__ float load(float v) const { return rd_clip(v); }
    __device__ __forceinline__ float term(float x, float y) const
    {
        if (x == 0.0f && y == 0.0f) return 0.0f;
        const float d = x - y;
        const float s = x + y + delta * fabsf(d);
        return __fdividef(d * (delta * fabsf(d) + x + 3.0f * y), s * s);
    }
};

struct TvGradOp {
    HuberP hb;
    bool p_is_one;
    __device__ __forceinline__ float load(float v) const { return v; }
    __device__ __forceinline__ float term(float x, float y) const
    {
        const float t = x - y;
        if (p_is_one) {  // p * slope * |t|^p / t = slope * sign(t) beyond delta
            const float a = fabsf(t);
            return a <= hb.delta ? t : copysignf(hb.slope, t);
        }
        return hb.dh(t);
    }
};

template <class Op>
__global__ void __launch_bounds__(STJ * STK)
k_grad_tiled(const float* __restrict__ f, float* __restrict__ Df, Dims d, Op op, float beta, int nbrs, bool planar)
{
    __shared__ float pl[3][SHJ][SHK];
    // 1-D blocks (block_sum indexes threads by threadIdx.x): tk fastest
    const int tid = threadIdx.x, tk = tid % STK, tj = tid / STK;
    const int k0 = blockIdx.x * STK, j0 = blockIdx.y * STJ;
    const int i0 = blockIdx.z * SPLANES, i1 = min(d.n1, i0 + SPLANES);
    const int k = k0 + tk, j = j0 + tj;
    // halo elements e = tid and tid + 256 of a plane: (hj, hk) in the
    // (SHJ x SHK) tile; a plane is fetched into registers one plane ahead
    // of its use (the global latency overlaps the current plane's stencil)
    constexpr int NE = (SHJ * SHK + STJ * STK - 1) / (STJ * STK);
    size_t off[NE];
    int hjk[NE];
#pragma unroll
    for (int q = 0; q < NE; q++) {
        const int e = tid + q * STJ * STK;
        const int hj = e / SHK, hk = e - hj * SHK;
        const int jj = min(d.n2 - 1, max(0, j0 + hj - 1)), kk = min(d.n3 - 1, max(0, k0 + hk - 1));
        off[q] = size_t(jj) * d.n3 + kk;
        hjk[q] = e < SHJ * SHK ? e : -1;
    }
    const size_t plane = size_t(d.n2) * d.n3;
    float v[NE];
    auto fetch = [&](int i) {
        const size_t b = size_t(min(d.n1 - 1, max(0, i))) * plane;
#pragma unroll
        for (int q = 0; q < NE; q++) v[q] = hjk[q] >= 0 ? op.load(__ldg(&f[b + off[q]])) : 0.0f;
    };
    auto store = [&](int slot) {
#pragma unroll
        for (int q = 0; q < NE; q++)
            if (hjk[q] >= 0) (&pl[slot][0][0])[hjk[q]] = v[q];
    };
    fetch(i0 - 1);
    store(0);
    fetch(i0);
    store(1);
    fetch(i0 + 1);
    int sm = 0, sc = 1, sp = 2;  // slots of planes i - 1, i, i + 1
    for (int i = i0; i < i1; i++) {
        store(sp);
        __syncthreads();
        if (i + 1 < i1) fetch(i + 2);
        if (j < d.n2 && k < d.n3) {
            const float x = pl[sc][tj + 1][tk + 1];
            float s[4] = {0.f, 0.f, 0.f, 0.f};
            const int slot3[3] = {sm, sc, sp};
#pragma unroll
            for (int di = -1; di <= 1; di++)
#pragma unroll
                for (int dj = -1; dj <= 1; dj++)
#pragma unroll
                    for (int dk = -1; dk <= 1; dk++) {
                        const int cls = (di != 0) + (dj != 0) + (dk != 0);
                        if (cls == 0) continue;
                        if (planar && di != 0) continue;  // N1 == 1: in-plane neighbours only
                        if (nbrs == 6 && cls > 1) continue;
                        s[cls] += op.term(x, pl[slot3[di + 1]][tj + 1 + dj][tk + 1 + dk]);
                    }
            Df[vidx(d, i, j, k)] = combine(s[1], s[2], s[3], beta);
        }
        __syncthreads();  // plane i - 1 is overwritten next
        const int t = sm;
        sm = sc;
        sc = sp;
        sp = t;
    }
}

// Costs (sums over voxels of a per-voxel stencil term) on the same tiles:
// each thread adds its voxels' terms in double in plane order, the CTA adds
// its threads in a fixed order into one partial per CTA, and a second pass
// adds the partials in CTA order: deterministic.  TWO: the quadratic form's
// second array (the direction d) is tiled beside f.
struct RdCostOp {
    float delta, beta;
    __device__ __forceinline__ float load(float v) const { return rd_clip(v); }
    template <class Nb>
    __device__ __forceinline__ double voxel(float x, float, Nb nb) const
    {
        double s[4] = {0, 0, 0, 0};
        nb([&](int cls, float y, float) { s[cls] += rd_pot(x, y, delta); });
        return s[1] * double(1.0f * beta) + s[2] * double(0.7071067811865475f * beta) +
               s[3] * double(0.5773502691896258f * beta);
    }
};

struct TvCostOp {
    HuberP hb;
    float beta;
    bool p_is_one;
    __device__ __forceinline__ float load(float v) const { return v; }
    template <class Nb>
    __device__ __forceinline__ double voxel(float x, float, Nb nb) const
    {
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        if (p_is_one) {  // slope * |t|^1 + shift beyond delta
            nb([&](int cls, float y, float) {
                const float t = x - y, a = fabsf(t);
                s[cls] += a <= hb.delta ? 0.5f * t * t : hb.slope * a + hb.shift;
            });
        } else {
            nb([&](int cls, float y, float) { s[cls] += hb.h(x - y); });
        }
        return double(combine(s[1], s[2], s[3], beta));
    }
};

struct TvQuadOp {
    HuberP hb;
    float beta;
    bool p_is_one;
    __device__ __forceinline__ float load(float v) const { return v; }
    template <class Nb>
    __device__ __forceinline__ double voxel(float x, float xd, Nb nb) const
    {
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        if (p_is_one) {  // p slope |t|^(p-2) = slope / |t| beyond delta
            nb([&](int cls, float y, float yd) {
                const float e = xd - yd, a = fabsf(x - y);
                s[cls] += (a <= hb.delta ? 1.0f : hb.slope / a) * e * e;
            });
        } else {
            nb([&](int cls, float y, float yd) {
                const float e = xd - yd;
                s[cls] += hb.ddh(x - y) * e * e;
            });
        }
        return double(combine(s[1], s[2], s[3], beta));
    }
};

template <class Op, bool TWO>
__global__ void __launch_bounds__(STJ * STK)
k_cost_tiled(const float* __restrict__ f, const float* __restrict__ g2, Dims d, Op op, int nbrs, bool planar,
             double* __restrict__ partial)
{
    __shared__ float pl[3][SHJ][SHK];
    __shared__ float pd[TWO ? 3 : 1][SHJ][SHK];
    // 1-D blocks (block_sum indexes threads by threadIdx.x): tk fastest
    const int tid = threadIdx.x, tk = tid % STK, tj = tid / STK;
    const int k0 = blockIdx.x * STK, j0 = blockIdx.y * STJ;
    const int i0 = blockIdx.z * SPLANES, i1 = min(d.n1, i0 + SPLANES);
    const int k = k0 + tk, j = j0 + tj;
    // planes fetched into registers one plane ahead of their use, as in
    // k_grad_tiled
    constexpr int NE = (SHJ * SHK + STJ * STK - 1) / (STJ * STK);
    size_t off[NE];
    int hjk[NE];
#pragma unroll
    for (int q = 0; q < NE; q++) {
        const int e = tid + q * STJ * STK;
        const int hj = e / SHK, hk = e - hj * SHK;
        const int jj = min(d.n2 - 1, max(0, j0 + hj - 1)), kk = min(d.n3 - 1, max(0, k0 + hk - 1));
        off[q] = size_t(jj) * d.n3 + kk;
        hjk[q] = e < SHJ * SHK ? e : -1;
    }
    const size_t plane = size_t(d.n2) * d.n3;
    float v[NE], vd[NE];
    auto fetch = [&](int i) {
        const size_t b = size_t(min(d.n1 - 1, max(0, i))) * plane;
#pragma unroll
        for (int q = 0; q < NE; q++) {
            v[q] = hjk[q] >= 0 ? op.load(__ldg(&f[b + off[q]])) : 0.0f;
            vd[q] = (TWO && hjk[q] >= 0) ? __ldg(&g2[b + off[q]]) : 0.0f;
        }
    };
    auto store = [&](int slot) {
#pragma unroll
        for (int q = 0; q < NE; q++)
            if (hjk[q] >= 0) {
                (&pl[slot][0][0])[hjk[q]] = v[q];
                if (TWO) (&pd[TWO ? slot : 0][0][0])[hjk[q]] = vd[q];
            }
    };
    fetch(i0 - 1);
    store(0);
    fetch(i0);
    store(1);
    fetch(i0 + 1);
    int sm = 0, sc = 1, sp = 2;
    double acc = 0.0;
    for (int i = i0; i < i1; i++) {
        store(sp);
        __syncthreads();
        if (i + 1 < i1) fetch(i + 2);
        if (j < d.n2 && k < d.n3) {
            const int slot3[3] = {sm, sc, sp};
            const float x = pl[sc][tj + 1][tk + 1];
            const float xd = TWO ? pd[TWO ? sc : 0][tj + 1][tk + 1] : 0.0f;
            acc += op.voxel(x, xd, [&](auto fn) {
#pragma unroll
                for (int di = -1; di <= 1; di++)
#pragma unroll
                    for (int dj = -1; dj <= 1; dj++)
#pragma unroll
                        for (int dk = -1; dk <= 1; dk++) {
                            const int cls = (di != 0) + (dj != 0) + (dk != 0);
                            if (cls == 0) continue;
                            if (planar && di != 0) continue;
                            if (nbrs == 6 && cls > 1) continue;
                            const int sl = slot3[di + 1];
                            fn(cls, pl[sl][tj + 1 + dj][tk + 1 + dk],
                               TWO ? pd[TWO ? sl : 0][tj + 1 + dj][tk + 1 + dk] : 0.0f);
                        }
            });
        }
        __syncthreads();
        const int t = sm;
        sm = sc;
        sc = sp;
        sp = t;
    }
    acc = block_sum<STJ * STK>(acc);
    if (tid == 0) partial[(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = acc;
}

template <class Op, bool TWO>
int cost_tiled(const float* f, const float* g2, const Dims& d, const Op& op, int nbrs, bool planar, double* out,
               cudaStream_t st, const char* name)
{
    dim3 block(STK * STJ, 1, 1), grid(ceil_div(d.n3, STK), ceil_div(d.n2, STJ), ceil_div(d.n1, SPLANES));
    const int nb = int(grid.x * grid.y * grid.z);
    double* part = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&part), sizeof(double) * nb, st));
    k_cost_tiled<Op, TWO><<<grid, block, 0, st>>>(f, g2, d, op, nbrs, planar, part);
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

bool dims_ok(int n1, int n2, int n3) { return n1 > 0 && n2 > 0 && n3 > 0 && n1 <= 65535; }

}  // namespace
}  // namespace petl

using namespace petl;

extern "C" {

int petl_rd_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, void* stream)
{
    PETL_REQUIRE(f && Df && dims_ok(N1, N2, N3), "rd_gradient: invalid arguments");
    const Dims d{N1, N2, N3};
    dim3 block(STK * STJ, 1, 1), grid(ceil_div(N3, STK), ceil_div(N2, STJ), ceil_div(N1, SPLANES));
    k_grad_tiled<RdGradOp><<<grid, block, 0, as_stream(stream)>>>(f, Df, d, RdGradOp{delta}, beta, 26, false);
    PETL_LAUNCH_CHECK("rd_gradient");
    return 0;
}

int petl_rd_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, double* out, void* stream)
{
    PETL_REQUIRE(f && out && dims_ok(N1, N2, N3), "rd_cost: invalid arguments");
    const Dims d{N1, N2, N3};
    return cost_tiled<RdCostOp, false>(f, nullptr, d, RdCostOp{delta, beta}, 26, false, out, as_stream(stream),
                                       "rd_cost");
}

int petl_tv_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, void* stream)
{
    PETL_REQUIRE(f && Df && dims_ok(N1, N2, N3), "tv_gradient: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    dim3 block(STK * STJ, 1, 1), grid(ceil_div(N3, STK), ceil_div(N2, STJ), ceil_div(N1, SPLANES));
    k_grad_tiled<TvGradOp><<<grid, block, 0, as_stream(stream)>>>(f, Df, d, TvGradOp{hb, p == 1.0f}, beta,
                                                                   numNeighbors == 6 ? 6 : 26, N1 == 1);
    PETL_LAUNCH_CHECK("tv_gradient");
    return 0;
}

int petl_tv_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, float p, int numNeighbors,
                     double* out, void* stream)
{
    PETL_REQUIRE(f && out && dims_ok(N1, N2, N3), "tv_cost: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    return cost_tiled<TvCostOp, false>(f, nullptr, d, TvCostOp{hb, beta, p == 1.0f}, numNeighbors == 6 ? 6 : 26, N1 == 1, out,
                                       as_stream(stream), "tv_cost");
}

int petl_tv_quadform_dev(const float* f, const float* dvec, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, double* out, void* stream)
{
    PETL_REQUIRE(f && dvec && out && dims_ok(N1, N2, N3), "tv_quadform: invalid arguments");
    const HuberP hb = make_huber(delta, beta, p);
    const Dims d{N1, N2, N3};
    return cost_tiled<TvQuadOp, true>(f, dvec, d, TvQuadOp{hb, beta, p == 1.0f}, numNeighbors == 6 ? 6 : 26, N1 == 1, out,
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
