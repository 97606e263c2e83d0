// Planogram corrections: the solid-angle scaling (src/planogram.cpp:262-302)
// and PETL::apply_corrections (src/petl.cpp:163-192), i.e. the division of
// the data by the response followed by the bad-pixel median in-fill of
// src/median_filter.cu:11-190.
//
// Solid angle: one factor per projection (iv1, iv0), computed on the host in
// double exactly as the reference's host code does (a table of N_v1 x N_v0
// floats), then one streaming multiply over the planogram: 8 bytes of HBM
// traffic per bin.
//
// apply_corrections: one CTA per projection (N_u1 x N_u0 bins).  The CTA
// stages the projection's response in shared memory, finds its median by a
// radix select over order-preserving keys (exact: the median is a value of
// the data, or the float mean of two), marks the bins whose response lies
// below rel * median, replaces the staged response by the divided data
// g / r, and writes every bin of the projection once:
//   outside the field of view -> 0
//   below the threshold       -> median of the 5x5 window's divided values
//                                that exceed the threshold
//   otherwise                 -> g / r
// 12 bytes of HBM traffic per bin (read r, read g, write g).  Projections
// larger than the shared-memory stage keep the divided values in a global
// scratch slice instead and read the response from HBM again.
//
// The reference kernel rewrites g in place while other threads of the same
// launch read their windows from it, so its result depends on thread order
// whenever a window holds a pixel that the launch rewrites; every window here
// reads the divided values as they were before any in-fill.  The reference
// tests a neighbour's divided value, not its response, against the threshold
// (its "r_proj" points into g); this kernel does the same.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "projector.cuh"

namespace petl {
namespace {

constexpr int kCorrThreads = 512;
constexpr int kCorrWarps = kCorrThreads / 32;
constexpr int kStageMax = 49152;  // bins of one projection staged in shared memory

// float -> unsigned key with the same order (negative values reversed)
__device__ __forceinline__ unsigned ordered_key(float x)
{
    const unsigned b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float key_value(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct SelectSmem {
    unsigned hist[kCorrWarps * 256];
    unsigned tot[256];
    unsigned bcast[2];
    unsigned red[2 * kCorrWarps];
};

__device__ __forceinline__ unsigned block_min_max(unsigned lo, unsigned hi, SelectSmem& s, unsigned* hi_out)
{
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __syncthreads();  // s.red may still be read by an earlier call
    if ((threadIdx.x & 31) == 0) {
        s.red[threadIdx.x >> 5] = lo;
        s.red[kCorrWarps + (threadIdx.x >> 5)] = hi;
    }
    __syncthreads();
    lo = 0xffffffffu;
    hi = 0;
    for (int w = 0; w < kCorrWarps; w++) {
        lo = min(lo, s.red[w]);
        hi = max(hi, s.red[kCorrWarps + w]);
    }
    *hi_out = hi;
    return lo;
}

// Key of rank k (0-based, ascending) among the n values x[0..n).  The bits
// that the smallest and largest keys share are common to all keys; the rest
// are resolved from the most significant end in digits of up to 8 bits, one
// pass over x per digit, with per-warp histograms in which same-digit lanes
// are combined (__match_any_sync) and warps with no candidate lane skip the
// combine.  *below_equal receives the number of values equal to the result
// that rank below k.
__device__ unsigned select_rank(const float* x, int n, unsigned k, SelectSmem& s, unsigned* below_equal)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned lo = 0xffffffffu, hi = 0;
    for (int i = threadIdx.x; i < n; i += kCorrThreads) {
        const unsigned key = ordered_key(x[i]);
        lo = min(lo, key);
        hi = max(hi, key);
    }
    lo = block_min_max(lo, hi, s, &hi);
    if (lo == hi) {
        *below_equal = k;
        return lo;
    }
    const int free_bits = 32 - __clz(lo ^ hi);
    unsigned prefix = free_bits == 32 ? 0u : (lo & (0xffffffffu << free_bits)), kk = k;
    const int nround = (n + kCorrThreads - 1) / kCorrThreads * kCorrThreads;
    for (int top = free_bits; top > 0; top -= 8) {
        const int shift = max(top - 8, 0);
        const unsigned above = top == 32 ? 0u : (0xffffffffu << top), dmask = (1u << (top - shift)) - 1u;
        for (int i = threadIdx.x; i < kCorrWarps * 256; i += kCorrThreads) s.hist[i] = 0;
        __syncthreads();
        unsigned* wh = s.hist + warp * 256;
        for (int i = threadIdx.x; i < nround; i += kCorrThreads) {
            unsigned d = 256;
            if (i < n) {
                const unsigned key = ordered_key(x[i]);
                if ((key & above) == prefix) d = (key >> shift) & dmask;
            }
            if (__any_sync(0xffffffffu, d < 256)) {
                const unsigned peers = __match_any_sync(0xffffffffu, d);
                if (d < 256 && lane == __ffs(peers) - 1) atomicAdd(&wh[d], unsigned(__popc(peers)));
            }
        }
        __syncthreads();
        if (threadIdx.x < 256) {
            unsigned t = 0;
            for (int w = 0; w < kCorrWarps; w++) t += s.hist[w * 256 + threadIdx.x];
            s.tot[threadIdx.x] = t;
        }
        __syncthreads();
        if (warp == 0) {
            unsigned c[8], sum = 0;
            for (int j = 0; j < 8; j++) {
                c[j] = s.tot[lane * 8 + j];
                sum += c[j];
            }
            unsigned incl = sum;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            unsigned before = incl - sum;
            for (int j = 0; j < 8; j++) {
                if (kk >= before && kk < before + c[j]) {
                    s.bcast[0] = prefix | (unsigned(lane * 8 + j) << shift);
                    s.bcast[1] = kk - before;
                }
                before += c[j];
            }
        }
        __syncthreads();
        prefix = s.bcast[0];
        kk = s.bcast[1];
    }
    *below_equal = kk;
    return prefix;
}

// Largest key below `bound` among x[0..n) (0 if none).
__device__ unsigned max_key_below(const float* x, int n, unsigned bound, SelectSmem& s)
{
    unsigned m = 0;
    for (int i = threadIdx.x; i < n; i += kCorrThreads) {
        const unsigned key = ordered_key(x[i]);
        if (key < bound && key > m) m = key;
    }
    unsigned mx;
    block_min_max(0xffffffffu, m, s, &mx);
    return mx;
}

// Median of x[0..n) as src/vector_ops.cpp:358-374 defines it: rank n/2, and
// for even n the float mean of ranks n/2 and n/2 - 1.
__device__ float block_median(const float* x, int n, SelectSmem& s)
{
    const unsigned mid = unsigned(n) / 2;
    unsigned eq_below = 0;
    const unsigned up = select_rank(x, n, mid, s, &eq_below);
    const float upper = key_value(up);
    if (n & 1) return upper;
    // rank mid - 1 equals rank mid when a copy of it ranks below mid
    const float lower = eq_below > 0 ? upper : key_value(max_key_below(x, n, up, s));
    return __fdiv_rn(__fadd_rn(upper, lower), 2.0f);
}

// Sorts 32 values held in registers (bitonic network, fully unrolled so that
// every index is a compile-time constant).
__device__ __forceinline__ void sort32(float (&v)[32])
{
#pragma unroll
    for (int ks = 1; ks <= 5; ks++)
#pragma unroll
        for (int js = ks - 1; js >= 0; js--)
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const int k = 1 << ks, l = i ^ (1 << js);
                if (l > i) {
                    const float a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? fminf(a, b) : fmaxf(a, b);
                    v[l] = up ? fmaxf(a, b) : fminf(a, b);
                }
            }
}

// Median of the values in the 5x5 window of (iu1, iu0) that exceed thr,
// rows and columns clamped at the projection's edges
// (src/median_filter.cu:57-118): 0 for none, the value for one, the float
// mean of the two middle values for an even count.  The window's values
// that do not exceed thr sort to the end as +inf.
__device__ __forceinline__ float window_fill(const float* d, int N1, int N0, int iu1, int iu0, float thr)
{
    float v[32];
    int m = 0;
#pragma unroll
    for (int dj = 0; dj < 5; dj++) {
        const int j = min(max(iu1 + dj - 2, 0), N1 - 1);
#pragma unroll
        for (int dk = 0; dk < 5; dk++) {
            const int i = min(max(iu0 + dk - 2, 0), N0 - 1);
            const float x = d[j * N0 + i];
            const bool ok = x > thr;
            v[dj * 5 + dk] = ok ? x : __int_as_float(0x7f800000);
            m += ok;
        }
    }
#pragma unroll
    for (int i = 25; i < 32; i++) v[i] = __int_as_float(0x7f800000);
    sort32(v);
    if (m == 0) return 0.0f;
    // v[h] and v[h-1] of the sorted values as a min / max over the ranks
    // (a reduction keeps v in registers; a picked index would not)
    const int h = m / 2;
    float a = __int_as_float(0x7f800000), b = __int_as_float(0xff800000);
#pragma unroll
    for (int i = 0; i < 25; i++) {
        a = fminf(a, i >= h ? v[i] : __int_as_float(0x7f800000));
        b = fmaxf(b, i < h ? v[i] : __int_as_float(0xff800000));
    }
    return (m & 1) ? a : __fmul_rn(0.5f, __fadd_rn(a, b));
}

struct CorrArgs {
    petl_geom G;
    float* g;
    const float* r;
    float* scratch;  // global path: one projection of divided values per CTA
    float rel;
    int view0, nviews;  // projections [view0, view0 + nviews)
};

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Persistent CTAs, one per SM, each correcting projections view0 + b,
// view0 + b + gridDim.x, ...  STAGE: the projection's response, then its
// divided values, live in shared memory next to a bitmask of the bins below
// the threshold; the bins are written in one pass (zero outside the field of
// view, g / r elsewhere) and the bins below the threshold are then
// overwritten with their window medians, spread evenly over the threads by
// their rank in the bitmask.  Otherwise (projections too large to stage) the
// divided values go to scratch + blockIdx.x * n and every bin is written
// once, in-filled where its response is below the threshold.
template <bool STAGE>
__global__ void __launch_bounds__(kCorrThreads, 1) k_apply_corrections(const CorrArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const petl_geom& G = a.G;
    const int N1 = G.N_u1, N0 = G.N_u0, n = N1 * N0;
    const int n4 = (n + 3) & ~3, nw = (n + 31) / 32;
    float* d = reinterpret_cast<float*>(smem_raw);
    unsigned* bad = reinterpret_cast<unsigned*>(d + n4);
    unsigned* rank = bad + nw + 1;
    SelectSmem& s = *reinterpret_cast<SelectSmem*>(STAGE ? reinterpret_cast<unsigned char*>(rank + nw + 1)
                                                         : smem_raw);
    // float4 paths need every projection 16-byte aligned
    const bool vec = (n & 3) == 0 && ((reinterpret_cast<uintptr_t>(a.g) | reinterpret_cast<uintptr_t>(a.r)) & 15) == 0;
    const size_t bytes = size_t(n) * 4;
    if (threadIdx.x == 0 && vec && blockIdx.x < a.nviews) {
        const size_t v = size_t(a.view0) + blockIdx.x;
        prefetch_l2(a.r + v * n, uint32_t(bytes));
        prefetch_l2(a.g + v * n, uint32_t(bytes));
    }
    for (int vi = blockIdx.x; vi < a.nviews; vi += gridDim.x) {
        const int view = a.view0 + vi;
        const int iv1 = view / G.N_v0, iv0 = view % G.N_v0;
        float* gv = a.g + size_t(view) * n;
        const float* rv = a.r + size_t(view) * n;
        if (threadIdx.x == 0 && vec && vi + gridDim.x < a.nviews) {
            const size_t nx = size_t(view) + gridDim.x;
            prefetch_l2(a.r + nx * n, uint32_t(bytes));
            prefetch_l2(a.g + nx * n, uint32_t(bytes));
        }
        float* dd = STAGE ? d : a.scratch + size_t(blockIdx.x) * n;
        if (STAGE) {
            if (vec) {
                const float4* r4 = reinterpret_cast<const float4*>(rv);
                float4* d4 = reinterpret_cast<float4*>(d);
#pragma unroll 8
                for (int i = threadIdx.x; i < n / 4; i += kCorrThreads) d4[i] = __ldcs(r4 + i);
            } else {
                for (int i = threadIdx.x; i < n; i += kCorrThreads) d[i] = __ldcs(rv + i);
            }
            __syncthreads();
        }
        const float thr = __fmul_rn(a.rel, block_median(STAGE ? d : rv, n, s));
        if (STAGE) {
            // bins below the threshold, one bit each
            const int nround = nw * 32;
            for (int i = threadIdx.x; i < ((nround + kCorrThreads - 1) / kCorrThreads) * kCorrThreads;
                 i += kCorrThreads) {
                const unsigned w = __ballot_sync(0xffffffffu, i < n && d[i] < thr);
                if ((threadIdx.x & 31) == 0 && i < nround) bad[i >> 5] = w;
            }
        }
        // divided values (src/data_cube.cpp:144-149)
        if (STAGE && vec) {
            const float4* g4 = reinterpret_cast<const float4*>(gv);
            float4* d4 = reinterpret_cast<float4*>(d);
#pragma unroll 4
            for (int i = threadIdx.x; i < n / 4; i += kCorrThreads) {
                const float4 x = __ldcs(g4 + i);
                float4 r = d4[i];
                r.x = (r.x == 0.0f) ? 0.0f : __fdiv_rn(x.x, r.x);
                r.y = (r.y == 0.0f) ? 0.0f : __fdiv_rn(x.y, r.y);
                r.z = (r.z == 0.0f) ? 0.0f : __fdiv_rn(x.z, r.z);
                r.w = (r.w == 0.0f) ? 0.0f : __fdiv_rn(x.w, r.w);
                d4[i] = r;
            }
        } else {
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const float r = STAGE ? d[i] : rv[i];
                dd[i] = (r == 0.0f) ? 0.0f : __fdiv_rn(__ldcs(gv + i), r);
            }
        }
        __syncthreads();
        if (!STAGE) {
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const int iu1 = i / N0, iu0 = i - iu1 * N0;
                float out;
                if (!ray_visible(G, iv1, iv0, iu1, iu0))
                    out = 0.0f;
                else
                    out = rv[i] < thr ? window_fill(dd, N1, N0, iu1, iu0, thr) : dd[i];
                __stcs(gv + i, out);
            }
            __syncthreads();  // the scratch slice is rewritten for the next projection
            continue;
        }
        // every bin: zero outside the field of view, else g / r
        if (vec) {
            float4* o4 = reinterpret_cast<float4*>(gv);
            for (int i4 = threadIdx.x; i4 < n / 4; i4 += kCorrThreads) {
                float4 x = reinterpret_cast<const float4*>(d)[i4];
                int iu1 = (4 * i4) / N0, iu0 = 4 * i4 - iu1 * N0;
                auto mask = [&](float& c) {
                    if (!ray_visible(G, iv1, iv0, iu1, iu0)) c = 0.0f;
                    if (++iu0 == N0) {
                        iu0 = 0;
                        iu1++;
                    }
                };
                mask(x.x);
                mask(x.y);
                mask(x.z);
                mask(x.w);
                __stcs(o4 + i4, x);
            }
        } else {
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const int iu1 = i / N0, iu0 = i - iu1 * N0;
                __stcs(gv + i, ray_visible(G, iv1, iv0, iu1, iu0) ? d[i] : 0.0f);
            }
        }
        // rank of the first bad bin of each bitmask word (exclusive scan)
        if (threadIdx.x < 32) {
            unsigned carry = 0;
            for (int w0 = 0; w0 < nw; w0 += 32) {
                const int w = w0 + threadIdx.x;
                const unsigned c = w < nw ? __popc(bad[w]) : 0u;
                unsigned incl = c;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (threadIdx.x >= o) incl += y;
                }
                if (w < nw) rank[w] = carry + incl - c;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (threadIdx.x == 0) rank[nw] = carry;
        }
        __syncthreads();  // orders the bulk writes above before the in-fill overwrites
        const unsigned nbad = rank[nw];
        for (unsigned q = threadIdx.x; q < nbad; q += kCorrThreads) {
            int lo = 0, hi = nw - 1;  // last word whose first rank is <= q
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (rank[mid] <= q) lo = mid; else hi = mid - 1;
            }
            const unsigned bit = __fns(bad[lo], 0, int(q - rank[lo]) + 1);
            const int i = lo * 32 + int(bit);
            if (bit >= 32 || i >= n) continue;  // not reached: q ranks a set bit of word lo
            const int iu1 = i / N0, iu0 = i - iu1 * N0;
            if (ray_visible(G, iv1, iv0, iu1, iu0)) __stcs(gv + i, window_fill(d, N1, N0, iu1, iu0, thr));
        }
        __syncthreads();  // shared memory is restaged for the next projection
    }
}

template <bool STAGE>
size_t corr_smem(int n)
{
    if (!STAGE) return sizeof(SelectSmem);
    const size_t nw = size_t(n + 31) / 32;
    return size_t((n + 3) & ~3) * 4 + (2 * nw + 2) * 4 + sizeof(SelectSmem);
}

__global__ void k_scale_views(float* g, const float* c, long long nviews, int view_elems, int vec4)
{
    for (long long v = blockIdx.y; v < nviews; v += gridDim.y) {
        const float f = c[v];
        float* p = g + v * view_elems;
        if (vec4) {
            float4* p4 = reinterpret_cast<float4*>(p);
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < view_elems / 4; i += gridDim.x * blockDim.x) {
                float4 x = __ldcs(p4 + i);
                x.x = __fmul_rn(x.x, f);
                x.y = __fmul_rn(x.y, f);
                x.z = __fmul_rn(x.z, f);
                x.w = __fmul_rn(x.w, f);
                __stcs(p4 + i, x);
            }
        } else {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < view_elems; i += gridDim.x * blockDim.x)
                p[i] = __fmul_rn(p[i], f);
        }
    }
}

bool v1_range_ok(const petl_geom& G, int b, int e) { return b >= 0 && e <= G.N_v1 && b <= e; }

// The corrections need the planogram only (no volume).
bool planogram_valid(const petl_geom& G, std::string* why)
{
    if (G.N_v1 <= 0 || G.N_v0 <= 0 || G.N_u1 <= 0 || G.N_u0 <= 0) {
        *why = "planogram not defined";
        return false;
    }
    if (!(G.T_v1 > 0.f) || !(G.T_v0 > 0.f) || !(G.T_u1 > 0.f) || !(G.T_u0 > 0.f)) {
        *why = "planogram pitch <= 0";
        return false;
    }
    if (double(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0 > 4.0e10 || double(G.N_u1) * G.N_u0 > 2.0e9) {
        *why = "array too large";
        return false;
    }
    return true;
}

}  // namespace

// The reference's per-projection factor (src/planogram.cpp:262-270, 290-293):
// v in float, 2 pi (1 + v0^2 + v1^2)^1.5 / (T_v1 T_v0) in double, rounded to
// float; the inverse is float(1.0 / c).  Host code compiled without
// floating-point contraction, as the reference's host code is.
std::vector<float> solid_angle_table(const petl_geom& G, bool inverse)
{
    std::vector<float> c(size_t(G.N_v1) * G.N_v0);
    for (int iv1 = 0; iv1 < G.N_v1; iv1++)
        for (int iv0 = 0; iv0 < G.N_v0; iv0++) {
            const float v1 = float(iv1) * G.T_v1 + G.v1_0;
            const float v0 = float(iv0) * G.T_v0 + G.v0_0;
            const double sq = 1.0 + double(v0 * v0) + double(v1 * v1);
            float f = float(2.0 * 3.1415926535897932385 * std::pow(sq, 1.5) / double(G.T_v1 * G.T_v0));
            if (inverse) f = float(1.0 / double(f));
            c[size_t(iv1) * G.N_v0 + iv0] = f;
        }
    return c;
}

// Scales projections iv1 in [iv1_b, iv1_e) of the planogram at g.
int solid_angle(const petl_geom& G, float* g, bool inverse, int iv1_b, int iv1_e, cudaStream_t st)
{
    std::string why;
    PETL_REQUIRE(planogram_valid(G, &why), "set_solid_angle_correction: " + why);
    PETL_REQUIRE(g != nullptr && v1_range_ok(G, iv1_b, iv1_e), "set_solid_angle_correction: invalid arguments");
    if (iv1_b == iv1_e) return 0;
    const std::vector<float> c = solid_angle_table(G, inverse);
    const long long v0 = (long long)iv1_b * G.N_v0, nviews = (long long)(iv1_e - iv1_b) * G.N_v0;
    const int ve = G.N_u1 * G.N_u0;
    float* gs = g + size_t(v0) * ve;
    const int vec4 = (ve & 3) == 0 && (reinterpret_cast<uintptr_t>(gs) & 15) == 0;
    float* dc = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&dc), size_t(nviews) * 4, st));
    cudaError_t e = cudaMemcpyAsync(dc, c.data() + v0, size_t(nviews) * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const unsigned per_view = unsigned(vec4 ? ve / 4 : ve);
        dim3 grid(std::max(1u, std::min(ceil_div(per_view, 256 * 4), 64u)), unsigned(std::min(nviews, 65535LL)));
        k_scale_views<<<grid, 256, 0, st>>>(gs, dc, nviews, ve, vec4);
        note_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(dc, st);
    if (e != cudaSuccess) {
        set_error(std::string("set_solid_angle_correction: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

// Corrects projections iv1 in [iv1_b, iv1_e) of the planogram at g with the
// response at r (both full planograms).
int apply_corrections(const petl_geom& G, float* g, const float* r, float rel, int iv1_b, int iv1_e,
                      cudaStream_t st)
{
    std::string why;
    PETL_REQUIRE(planogram_valid(G, &why), "apply_corrections: " + why);
    PETL_REQUIRE(g && r && v1_range_ok(G, iv1_b, iv1_e), "apply_corrections: invalid arguments");
    const int n = G.N_u1 * G.N_u0;
    const int first = iv1_b * G.N_v0, nviews = (iv1_e - iv1_b) * G.N_v0;
    if (nviews == 0) return 0;
    CorrArgs a{G, g, r, nullptr, rel, first, nviews};
    const int grid = std::min(nviews, sm_count());
    if (n <= kStageMax) {
        static int attr_set[64] = {0};
        int dev = 0;
        PETL_CUDA(cudaGetDevice(&dev));
        if (dev >= 0 && dev < 64 && !attr_set[dev]) {
            PETL_CUDA(cudaFuncSetAttribute(k_apply_corrections<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(corr_smem<true>(kStageMax))));
            attr_set[dev] = 1;
        }
        k_apply_corrections<true><<<grid, kCorrThreads, corr_smem<true>(n), st>>>(a);
        PETL_LAUNCH_CHECK("apply_corrections");
        return 0;
    }
    // large projections: divided values in a scratch slice per CTA
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&a.scratch), size_t(grid) * n * 4, st));
    k_apply_corrections<false><<<grid, kCorrThreads, corr_smem<false>(n), st>>>(a);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(a.scratch, st);
    if (e != cudaSuccess) {
        set_error(std::string("apply_corrections launch: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl

extern "C" {

int petl_solid_angle_dev(const petl_geom* G, float* g, int do_inverse, void* stream)
{
    PETL_REQUIRE(G != nullptr, "set_solid_angle_correction: null geometry");
    return petl::solid_angle(*G, g, do_inverse != 0, 0, G->N_v1, petl::as_stream(stream));
}

int petl_apply_corrections_dev(const petl_geom* G, float* g, const float* r, float threshold, void* stream)
{
    PETL_REQUIRE(G != nullptr, "apply_corrections: null geometry");
    return petl::apply_corrections(*G, g, r, threshold, 0, G->N_v1, petl::as_stream(stream));
}

}  // extern "C"
