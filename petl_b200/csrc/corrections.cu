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
constexpr int kStageMax = 45056;  // bins of one projection staged in shared memory
constexpr int kDigitBits = 12;    // width of the median search's first histogram
constexpr int kListMax = 2048;    // keys of the median's buckets resolved from a list

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
    unsigned hist[1 << kDigitBits];
    unsigned list[kListMax];
    unsigned red[2 * kCorrWarps];
    unsigned bcast[8];
    int box[4];  // visible columns [box0, box1] and rows [box2, box3] of the projection
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

// Exclusive prefix sum of v over the block's threads; *total gets the sum.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, SelectSmem& s, unsigned* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __syncthreads();  // s.red may still be read by an earlier call
    if (lane == 31) s.red[warp] = incl;
    __syncthreads();
    unsigned before = 0, tot = 0;
    for (int w = 0; w < kCorrWarps; w++) {
        const unsigned t = s.red[w];
        before += w < warp ? t : 0u;
        tot += t;
    }
    *total = tot;
    return before + incl - v;
}

// Bins of a histogram holding ranks ka and kb (kb <= ka): bcast[0] = bin of
// ka, bcast[1] = rank of ka inside it, bcast[2] = bin of kb, bcast[3] =
// number of keys in the bins below kb's.
__device__ void locate_ranks(const unsigned* hist, int nbins, unsigned ka, unsigned kb, SelectSmem& s)
{
    const int per = (nbins + kCorrThreads - 1) / kCorrThreads, b0 = threadIdx.x * per;
    unsigned sum = 0;
    for (int j = 0; j < per; j++)
        if (b0 + j < nbins) sum += hist[b0 + j];
    unsigned total;
    unsigned before = block_exclusive_scan(sum, s, &total);
    for (int j = 0; j < per && b0 + j < nbins; j++) {
        const unsigned c = hist[b0 + j];
        if (ka >= before && ka < before + c) {
            s.bcast[0] = b0 + j;
            s.bcast[1] = ka - before;
        }
        if (kb >= before && kb < before + c) {
            s.bcast[2] = b0 + j;
            s.bcast[3] = before;
        }
        before += c;
    }
    __syncthreads();
}

// Key of rank k among the n keys key_at(0..n), all of which share with
// `prefix` the bits at and above `top`: bits [0, top) are resolved from the
// most significant end in digits of up to 8 bits, one pass per digit, lanes
// with the same digit combined (__match_any_sync) and warps without a
// candidate skipping the combine.  *below_equal receives the number of keys
// equal to the result that rank below k.
template <class KeyAt>
__device__ unsigned radix_rank(KeyAt key_at, int n, unsigned prefix, int top, unsigned k, SelectSmem& s,
                               unsigned* below_equal)
{
    const int lane = threadIdx.x & 31;
    const int nround = (n + kCorrThreads - 1) / kCorrThreads * kCorrThreads;
    unsigned kk = k;
    for (; top > 0; top -= 8) {
        const int shift = max(top - 8, 0);
        const unsigned above = top == 32 ? 0u : (0xffffffffu << top), dmask = (1u << (top - shift)) - 1u;
        __syncthreads();  // the histogram may still be read by an earlier step
        for (int i = threadIdx.x; i < 256; i += kCorrThreads) s.hist[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < nround; i += kCorrThreads) {
            unsigned d = 256;
            if (i < n) {
                const unsigned key = key_at(i);
                if ((key & above) == prefix) d = (key >> shift) & dmask;
            }
            if (__any_sync(0xffffffffu, d < 256)) {
                const unsigned peers = __match_any_sync(0xffffffffu, d);
                if (d < 256 && lane == __ffs(peers) - 1) atomicAdd(&s.hist[d], unsigned(__popc(peers)));
            }
        }
        __syncthreads();
        locate_ranks(s.hist, 256, kk, kk, s);
        prefix |= s.bcast[0] << shift;
        kk = s.bcast[1];
    }
    *below_equal = kk;
    return prefix;
}

// Largest key below `bound` among key_at(0..n) (0 if none).
template <class KeyAt>
__device__ unsigned max_key_below(KeyAt key_at, int n, unsigned bound, SelectSmem& s)
{
    unsigned m = 0;
    for (int i = threadIdx.x; i < n; i += kCorrThreads) {
        const unsigned key = key_at(i);
        if (key < bound && key > m) m = key;
    }
    unsigned mx;
    block_min_max(0xffffffffu, m, s, &mx);
    return mx;
}

__device__ __forceinline__ float mean2(unsigned a, unsigned b)
{
    return __fdiv_rn(__fadd_rn(key_value(a), key_value(b)), 2.0f);
}

// Median of the n floats val(0..n) as src/vector_ops.cpp:358-374 defines
// it (rank n/2; for even n the float mean of ranks n/2 and n/2 - 1), given
// the smallest and largest of their keys.  One histogram pass over the top
// kDigitBits bits that the keys do not all share finds the buckets of the
// two ranks; a second pass lists the keys of those buckets, and the ranks
// are resolved on the list (on all keys if the list overflows).
template <class ValAt>
__device__ float block_median(ValAt val, int n, unsigned lo, unsigned hi, SelectSmem& s)
{
    const unsigned mid = unsigned(n) / 2;
    const bool even = (n & 1) == 0;
    if (lo == hi) return even ? mean2(lo, lo) : key_value(lo);
    const int lane = threadIdx.x & 31;
    const int free_bits = 32 - __clz(lo ^ hi);
    const unsigned common = free_bits == 32 ? 0u : (lo & (0xffffffffu << free_bits));
    const int dbits = min(kDigitBits, free_bits), shift = free_bits - dbits;
    const unsigned dmask = (1u << dbits) - 1u;
    const int nround = (n + kCorrThreads - 1) / kCorrThreads * kCorrThreads;
    for (int i = threadIdx.x; i < (1 << dbits); i += kCorrThreads) s.hist[i] = 0;
    if (threadIdx.x == 0) s.bcast[4] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nround; i += kCorrThreads) {
        const unsigned d = i < n ? (ordered_key(val(i)) >> shift) & dmask : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (i < n && lane == __ffs(peers) - 1) atomicAdd(&s.hist[d], unsigned(__popc(peers)));
    }
    __syncthreads();
    locate_ranks(s.hist, 1 << dbits, mid, even ? mid - 1 : mid, s);
    const unsigned b_up = s.bcast[0], b_lo = s.bcast[2], base = s.bcast[3];
    for (int i = threadIdx.x; i < nround; i += kCorrThreads) {
        unsigned key = 0;
        bool take = false;
        if (i < n) {
            key = ordered_key(val(i));
            const unsigned d = (key >> shift) & dmask;
            take = d >= b_lo && d <= b_up;
        }
        const unsigned m = __ballot_sync(0xffffffffu, take);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned pos0 = 0;
            if (lane == leader) pos0 = atomicAdd(&s.bcast[4], unsigned(__popc(m)));
            pos0 = __shfl_sync(0xffffffffu, pos0, leader);
            const unsigned pos = pos0 + __popc(m & ((1u << lane) - 1u));
            if (take && pos < kListMax) s.list[pos] = key;
        }
    }
    __syncthreads();
    const unsigned cnt = s.bcast[4];
    unsigned eq_below, up, low;
    if (cnt <= kListMax) {
        auto listed = [&](int i) { return s.list[i]; };
        up = radix_rank(listed, int(cnt), common, free_bits, mid - base, s, &eq_below);
        if (!even) return key_value(up);
        low = eq_below > 0 ? up : max_key_below(listed, int(cnt), up, s);
    } else {
        auto keyed = [&](int i) { return ordered_key(val(i)); };
        up = radix_rank(keyed, n, common, free_bits, mid, s, &eq_below);
        if (!even) return key_value(up);
        low = eq_below > 0 ? up : max_key_below(keyed, n, up, s);
    }
    return mean2(up, low);
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

__device__ __forceinline__ float divided(float g, float r) { return (r == 0.0f) ? 0.0f : __fdiv_rn(g, r); }

// Persistent CTAs, one per SM, each correcting projections view0 + b,
// view0 + b + gridDim.x, ... while the next one is prefetched into L2.
// Per projection: the visible columns and rows (two intervals), the
// response's key range, its median, then
//   STAGE: the response is staged in shared memory and replaced by the
//   divided values while a bitmask records the bins below the threshold;
//   every bin is written once (zero outside the field of view, g / r
//   inside) and the visible bins below the threshold are then overwritten
//   with their window medians, spread evenly over the threads by their rank
//   in the bitmask;
//   otherwise (projections too large to stage): the divided values go to
//   scratch + blockIdx.x * n and every bin is written once.
template <bool STAGE>
__global__ void __launch_bounds__(kCorrThreads, 1) k_apply_corrections(const CorrArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const petl_geom& G = a.G;
    const int N1 = G.N_u1, N0 = G.N_u0, n = N1 * N0;
    const int n4 = (n + 3) & ~3, nw = (n + 31) / 32;
    const int lane = threadIdx.x & 31;
    float* d = reinterpret_cast<float*>(smem_raw);
    unsigned* bad = reinterpret_cast<unsigned*>(d + n4);
    unsigned* rank = bad + nw + 1;
    SelectSmem& s = *reinterpret_cast<SelectSmem*>(STAGE ? reinterpret_cast<unsigned char*>(rank + nw + 1)
                                                         : smem_raw);
    // float4 paths: rows of whole float4s, every projection 16-byte aligned
    const bool vec =
        (N0 & 3) == 0 && ((reinterpret_cast<uintptr_t>(a.g) | reinterpret_cast<uintptr_t>(a.r)) & 15) == 0;
    const uint32_t bytes = uint32_t(n) * 4u;
    if (threadIdx.x == 0 && vec && blockIdx.x < a.nviews) {
        const size_t v = size_t(a.view0) + blockIdx.x;
        prefetch_l2(a.r + v * n, bytes);
        prefetch_l2(a.g + v * n, bytes);
    }
    for (int vi = blockIdx.x; vi < a.nviews; vi += gridDim.x) {
        const int view = a.view0 + vi;
        const int iv1 = view / G.N_v0, iv0 = view % G.N_v0;
        float* gv = a.g + size_t(view) * n;
        const float* rv = a.r + size_t(view) * n;
        if (threadIdx.x == 0) {
            if (vec && vi + gridDim.x < a.nviews) {
                const size_t nx = size_t(view) + gridDim.x;
                prefetch_l2(a.r + nx * n, bytes);
                prefetch_l2(a.g + nx * n, bytes);
            }
            s.box[0] = N0;
            s.box[1] = -1;
            s.box[2] = N1;
            s.box[3] = -1;
        }
        // the response (staged) and its key range
        unsigned lo = 0xffffffffu, hi = 0;
        if (STAGE && vec) {
            const float4* r4 = reinterpret_cast<const float4*>(rv);
            float4* d4 = reinterpret_cast<float4*>(d);
#pragma unroll 4
            for (int i = threadIdx.x; i < n / 4; i += kCorrThreads) {
                const float4 x = __ldcs(r4 + i);
                d4[i] = x;
                const unsigned k0 = ordered_key(x.x), k1 = ordered_key(x.y), k2 = ordered_key(x.z),
                               k3 = ordered_key(x.w);
                lo = min(min(lo, min(k0, k1)), min(k2, k3));
                hi = max(max(hi, max(k0, k1)), max(k2, k3));
            }
        } else {
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const float x = __ldcs(rv + i);
                if (STAGE) d[i] = x;
                lo = min(lo, ordered_key(x));
                hi = max(hi, ordered_key(x));
            }
        }
        lo = block_min_max(lo, hi, s, &hi);  // (its barriers also publish the stage and the box reset)
        for (int c = threadIdx.x; c < N0; c += kCorrThreads)
            if (u0_visible(G, iv0, c)) {
                atomicMin(&s.box[0], c);
                atomicMax(&s.box[1], c);
            }
        for (int r = threadIdx.x; r < N1; r += kCorrThreads)
            if (u1_visible(G, iv1, r)) {
                atomicMin(&s.box[2], r);
                atomicMax(&s.box[3], r);
            }
        __syncthreads();  // the box is read below (the median may take no barrier)
        float med;
        if (STAGE)
            med = block_median([&](int i) { return d[i]; }, n, lo, hi, s);
        else
            med = block_median([&](int i) { return rv[i]; }, n, lo, hi, s);
        const float thr = __fmul_rn(a.rel, med);
        const int c0 = s.box[0], c1 = s.box[1], r0 = s.box[2], r1 = s.box[3];
        auto visible = [&](int row, int col) { return col >= c0 && col <= c1 && row >= r0 && row <= r1; };

        if (!STAGE) {
            float* dd = a.scratch + size_t(blockIdx.x) * n;
            for (int i = threadIdx.x; i < n; i += kCorrThreads) dd[i] = divided(__ldcs(gv + i), rv[i]);
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const int row = i / N0, col = i - row * N0;
                float out = 0.0f;
                if (visible(row, col)) out = rv[i] < thr ? window_fill(dd, N1, N0, row, col, thr) : dd[i];
                __stcs(gv + i, out);
            }
            __syncthreads();  // the scratch slice is rewritten for the next projection
            continue;
        }
        // divided values in place of the response, and the bitmask of the
        // bins below the threshold (src/data_cube.cpp:144-149)
        if (vec) {
            const float4* g4 = reinterpret_cast<const float4*>(gv);
            float4* d4 = reinterpret_cast<float4*>(d);
            const int q4 = n / 4, qround = (q4 + kCorrThreads - 1) / kCorrThreads * kCorrThreads;
#pragma unroll 2
            for (int i4 = threadIdx.x; i4 < qround; i4 += kCorrThreads) {
                unsigned nib = 0;
                if (i4 < q4) {
                    const float4 x = __ldcs(g4 + i4);
                    float4 r = d4[i4];
                    nib = unsigned(r.x < thr) | unsigned(r.y < thr) << 1 | unsigned(r.z < thr) << 2 |
                          unsigned(r.w < thr) << 3;
                    r.x = divided(x.x, r.x);
                    r.y = divided(x.y, r.y);
                    r.z = divided(x.z, r.z);
                    r.w = divided(x.w, r.w);
                    d4[i4] = r;
                }
                // lanes 8j..8j+7 hold the 32 bins of one bitmask word
                unsigned w = nib << (4 * (lane & 7));
                w |= __shfl_xor_sync(0xffffffffu, w, 1);
                w |= __shfl_xor_sync(0xffffffffu, w, 2);
                w |= __shfl_xor_sync(0xffffffffu, w, 4);
                if ((lane & 7) == 0 && i4 < q4) bad[i4 >> 3] = w;
            }
        } else {
            const int nround = nw * 32, iround = (nround + kCorrThreads - 1) / kCorrThreads * kCorrThreads;
            for (int i = threadIdx.x; i < iround; i += kCorrThreads) {
                const bool b = i < n && d[i] < thr;
                if (i < n) d[i] = divided(__ldcs(gv + i), d[i]);
                const unsigned w = __ballot_sync(0xffffffffu, b);
                if (lane == 0 && i < nround) bad[i >> 5] = w;
            }
        }
        __syncthreads();
        // every bin: zero outside the field of view, g / r inside
        if (vec) {
            const float4* d4 = reinterpret_cast<const float4*>(d);
            float4* o4 = reinterpret_cast<float4*>(gv);
            const int step = 4 * kCorrThreads, drow = step / N0, dcol = step - drow * N0;
            int row = (4 * threadIdx.x) / N0, col = 4 * threadIdx.x - row * N0;
            for (int i4 = threadIdx.x; i4 < n / 4; i4 += kCorrThreads) {
                float4 x = d4[i4];
                if (!(row >= r0 && row <= r1)) {
                    x = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                } else {
                    x.x = (col >= c0 && col <= c1) ? x.x : 0.0f;
                    x.y = (col + 1 >= c0 && col + 1 <= c1) ? x.y : 0.0f;
                    x.z = (col + 2 >= c0 && col + 2 <= c1) ? x.z : 0.0f;
                    x.w = (col + 3 >= c0 && col + 3 <= c1) ? x.w : 0.0f;
                }
                __stcs(o4 + i4, x);
                row += drow;
                col += dcol;
                if (col >= N0) {
                    col -= N0;
                    row++;
                }
            }
        } else {
            for (int i = threadIdx.x; i < n; i += kCorrThreads) {
                const int row = i / N0, col = i - row * N0;
                __stcs(gv + i, visible(row, col) ? d[i] : 0.0f);
            }
        }
        // rank of the first bin below the threshold in each bitmask word
        const int per = (nw + kCorrThreads - 1) / kCorrThreads, w0 = threadIdx.x * per;
        unsigned cnt = 0;
        for (int j = 0; j < per; j++)
            if (w0 + j < nw) cnt += __popc(bad[w0 + j]);
        unsigned nbad;
        unsigned before = block_exclusive_scan(cnt, s, &nbad);
        for (int j = 0; j < per; j++)
            if (w0 + j < nw) {
                rank[w0 + j] = before;
                before += __popc(bad[w0 + j]);
            }
        __syncthreads();  // (also orders the bulk writes above before the in-fill overwrites)
        for (unsigned q = threadIdx.x; q < nbad; q += kCorrThreads) {
            int wlo = 0, whi = nw - 1;  // last word whose first rank is <= q
            while (wlo < whi) {
                const int m = (wlo + whi + 1) >> 1;
                if (rank[m] <= q)
                    wlo = m;
                else
                    whi = m - 1;
            }
            const unsigned bit = __fns(bad[wlo], 0, int(q - rank[wlo]) + 1);
            const int i = wlo * 32 + int(bit);
            if (bit >= 32 || i >= n) continue;  // not reached: q ranks a set bit of word wlo
            const int row = i / N0, col = i - row * N0;
            if (visible(row, col)) __stcs(gv + i, window_fill(d, N1, N0, row, col, thr));
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
