// PFDR rebinning, ramp filter and FBP.
//
// PFDR (reference src/pfdr.cu:43-315).  The reference zero-pads every
// (v1, u1) slice to NY x NX = optimalFFTsize(N_v0) x optimalFFTsize(N_u0),
// takes a 2-D R2C transform, accumulates over v1 the spectra whose
// u0-frequency passes the mask  |v1| <= T_v1/2  or  |U| > |v1|/(4 T_u1 v_m0)
// (the oblique u1 index of line 107 is u1 itself, so no sample moves),
// normalises by 1/(NY*NX*count(U)) (count not applied at U = 0), inverts
// with a 2-D C2R and crops.  The mask and the normalisation depend only on
// the u0-frequency, so the transform along v0 is applied and then exactly
// undone; it contributes nothing but a factor NY.  This file therefore runs
// the same arithmetic with 1-D transforms along u0 only: one pass over the
// planogram, every row transformed once, spectra accumulated in shared
// memory, one inverse transform per output row.  Transforms are hand-written
// mixed radix-4/2/3 Stockham FFTs in shared memory (all optimalFFTsize values
// are 2^a 3^b).  The masks, counts and per-row weights are computed on the
// host with the reference's float expressions.
//
// Ramp filter (src/ramp_filter.cu:24-76,156-348).  The reference multiplies
// the zero-padded (N_H >= 2 N_u0) row spectrum by Re(FFT(h))/N_H with
// h[s] = 1/(T pi (1/4 - s^2)); since h is circularly symmetric and the
// padding leaves no wrap-around, that is exactly the linear convolution of
// the row with h.  It is computed here as a direct convolution in shared
// memory (N_u0^2 FMAs per row, a few microseconds for the whole planogram),
// fused with the inverse planogram weight that PETL::doFBP applies next
// (src/planogram.cpp:304-333).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "projector.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {

int dispatch_mode();

namespace {

constexpr int kPfdrRows = 8;     // planogram rows (u1) per CTA, packed two per complex FFT
constexpr int kPfdrThreads = 128;
constexpr int kMaxFFT = 2048;
constexpr int kMaxStages = 12;

struct FFTPlan {
    int n;
    int nstages;
    int radix[kMaxStages];
};

FFTPlan make_plan(int n)
{
    FFTPlan p{};
    p.n = n;
    int m = n;
    while (m % 4 == 0) { p.radix[p.nstages++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.nstages++] = 2; m /= 2; }
    while (m % 3 == 0) { p.radix[p.nstages++] = 3; m /= 3; }
    p.nstages = m == 1 ? p.nstages : -1;
    return p;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Batched complex FFTs of length plan.n on nb contiguous sequences in shared
// memory.  'a' holds the input and receives the output (b is scratch).
// tw[m] = exp(-2 pi i m / n); sign = -1 forward, +1 inverse (unnormalised).
__device__ void smem_fft(float2* a, float2* b, const float2* tw, const FFTPlan& plan, int nb, int sign)
{
    const int n = plan.n;
    int Ns = 1;
    float2* src = a;
    float2* dst = b;
    for (int s = 0; s < plan.nstages; s++) {
        const int R = plan.radix[s];
        const int nbf = n / R;
        const int twstep = n / (Ns * R);
        for (int t = threadIdx.x; t < nb * nbf; t += blockDim.x) {
            const int seq = t / nbf, j = t - seq * nbf;
            const float2* in = src + seq * n;
            float2* out = dst + seq * n;
            const int k = j % Ns;
            float2 v[4];
            for (int r = 0; r < R; r++) {
                float2 x = in[j + r * nbf];
                if (r && k) {
                    float2 w = tw[(r * k * twstep) % n];
                    w.y *= float(-sign);  // tw is the forward table; conjugate for the inverse
                    x = cmul(x, w);
                }
                v[r] = x;
            }
            float2 V[4];
            if (R == 2) {
                V[0] = make_float2(v[0].x + v[1].x, v[0].y + v[1].y);
                V[1] = make_float2(v[0].x - v[1].x, v[0].y - v[1].y);
            } else if (R == 4) {
                const float2 s02 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
                const float2 d02 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
                const float2 s13 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
                const float2 d13 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
                // multiply d13 by (sign * i)
                const float2 jd13 = make_float2(-float(sign) * d13.y, float(sign) * d13.x);
                V[0] = make_float2(s02.x + s13.x, s02.y + s13.y);
                V[2] = make_float2(s02.x - s13.x, s02.y - s13.y);
                V[1] = make_float2(d02.x + jd13.x, d02.y + jd13.y);
                V[3] = make_float2(d02.x - jd13.x, d02.y - jd13.y);
            } else {  // R == 3
                const float c = -0.5f, sn = float(sign) * 0.86602540378443864676f;
                const float2 s12 = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
                const float2 d12 = make_float2(v[1].x - v[2].x, v[1].y - v[2].y);
                V[0] = make_float2(v[0].x + s12.x, v[0].y + s12.y);
                const float2 m = make_float2(v[0].x + c * s12.x, v[0].y + c * s12.y);
                // sn * i * d12
                const float2 jd = make_float2(-sn * d12.y, sn * d12.x);
                V[1] = make_float2(m.x + jd.x, m.y + jd.y);
                V[2] = make_float2(m.x - jd.x, m.y - jd.y);
            }
            const int idx = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; r++) out[idx + r * Ns] = V[r];
        }
        __syncthreads();
        float2* tmp = src;
        src = dst;
        dst = tmp;
        Ns *= R;
    }
    // result must end in 'a'
    if (src != a) {
        for (int t = threadIdx.x; t < nb * n; t += blockDim.x) a[t] = src[t];
        __syncthreads();
    }
}

struct PfdrArgs {
    const float* g;
    float* g_reb;
    int N_v1, N_v0, N_u1, N_u0;
    int NX;
    const float* row_w;    // [N_v1][N_v0] 1/sqrt(1+v1^2+v0^2)
    const float* absU;     // [NXH] |U(i)|
    const float* v1ap;     // [N_v1] |v1| * apertureConstant
    const unsigned char* central;  // [N_v1] |v1| <= T_v1/2
    const float* norm;     // [NXH] 1/(NX * count(U)) (count omitted at U = 0)
    const float* out_w;    // [N_v0] sqrt(1+v0^2)
    const float2* tw;      // [NX] forward twiddles
    FFTPlan plan;
    // streamed kernel: slices in processing order and the groups of one or
    // two slices transformed together (slopes +v1 and -v1 share the mask and
    // the normalisation, so their weighted rows are added before one
    // transform: the transform is linear)
    const int* order;      // [N_v1] slice of each load position
    const int* gfirst;     // [ngroups + 1] first load position of each group
    int ngroups;
};

__global__ void __launch_bounds__(kPfdrThreads) k_pfdr(const PfdrArgs A)
{
    extern __shared__ float2 sm[];
    const int NX = A.NX, NXH = NX / 2 + 1;
    constexpr int NB = kPfdrRows / 2;  // complex sequences
    float2* buf = sm;                  // NB * NX
    float2* tmp = buf + NB * NX;       // NB * NX
    float2* acc = tmp + NB * NX;       // kPfdrRows * NXH
    float2* tw = acc + kPfdrRows * NXH;  // NX
    float* absU = reinterpret_cast<float*>(tw + NX);  // NXH
    const int iv0 = blockIdx.x;
    const int iu1_0 = blockIdx.y * kPfdrRows;
    const int nrows = min(kPfdrRows, A.N_u1 - iu1_0);
    for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = A.tw[i];
    for (int i = threadIdx.x; i < NXH; i += blockDim.x) absU[i] = A.absU[i];
    for (int i = threadIdx.x; i < kPfdrRows * NXH; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
    __syncthreads();
    const size_t slab = size_t(A.N_v0) * A.N_u1 * A.N_u0;
    for (int iv1 = 0; iv1 < A.N_v1; iv1++) {
        const float w = A.row_w[iv1 * A.N_v0 + iv0];
        const float* src = A.g + iv1 * slab + (size_t(iv0) * A.N_u1 + iu1_0) * A.N_u0;
        // rows 2q (real part) and 2q+1 (imaginary part) of sequence q
        for (int t = threadIdx.x; t < NB * NX; t += blockDim.x) {
            const int q = t / NX, i = t - q * NX;
            float re = 0.f, im = 0.f;
            if (i < A.N_u0) {
                if (2 * q < nrows) re = __ldg(&src[size_t(2 * q) * A.N_u0 + i]) * w;
                if (2 * q + 1 < nrows) im = __ldg(&src[size_t(2 * q + 1) * A.N_u0 + i]) * w;
            }
            buf[t] = make_float2(re, im);
        }
        __syncthreads();
        smem_fft(buf, tmp, tw, A.plan, NB, -1);
        // split the two real spectra and accumulate the masked bins
        const bool cen = A.central[iv1] != 0;
        const float thr = A.v1ap[iv1];
        for (int t = threadIdx.x; t < NB * NXH; t += blockDim.x) {
            const int q = t / NXH, k = t - q * NXH;
            if (!(cen || absU[k] > thr)) continue;
            const float2 z = buf[q * NX + k];
            const float2 zc = buf[q * NX + (k == 0 ? 0 : NX - k)];
            // X0 = (Z + conj(Zc))/2, X1 = (Z - conj(Zc))/(2i)
            const float2 x0 = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
            const float2 x1 = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
            float2& a0 = acc[(2 * q) * NXH + k];
            float2& a1 = acc[(2 * q + 1) * NXH + k];
            a0.x += x0.x; a0.y += x0.y;
            a1.x += x1.x; a1.y += x1.y;
        }
        __syncthreads();
    }
    // normalise and pack pairs of rows into one inverse transform
    for (int t = threadIdx.x; t < NB * NX; t += blockDim.x) {
        const int q = t / NX, k = t - q * NX;
        const int kk = k <= NX / 2 ? k : NX - k;
        float2 a = acc[(2 * q) * NXH + kk], b = acc[(2 * q + 1) * NXH + kk];
        const float nr = A.norm[kk];
        a.x *= nr; a.y *= nr; b.x *= nr; b.y *= nr;
        if (kk == 0 || 2 * kk == NX) { a.y = 0.f; b.y = 0.f; }  // C2R ignores these
        if (k > NX / 2) { a.y = -a.y; b.y = -b.y; }             // Hermitian extension
        buf[t] = make_float2(a.x - b.y, a.y + b.x);             // A + iB
    }
    __syncthreads();
    smem_fft(buf, tmp, tw, A.plan, NB, +1);
    const float ow = A.out_w[iv0];
    for (int t = threadIdx.x; t < nrows * A.N_u0; t += blockDim.x) {
        const int r = t / A.N_u0, i = t - r * A.N_u0;
        const float2 z = buf[(r >> 1) * NX + i];
        const float v = (r & 1) ? z.y : z.x;
        A.g_reb[(size_t(iv0) * A.N_u1 + iu1_0 + r) * A.N_u0 + i] = v * ow;
    }
}

// ---------------------------------------------------------------------------
// Streamed PFDR for power-of-two transform sizes and rows of a multiple of 4
// floats (the workload sizes: N_u0 = 128 / 256 -> NX = 128 / 256).  Same
// arithmetic as k_pfdr, organised for bandwidth:
//  * a CTA owns kPfdrRows planogram rows (u1) of one view v0 and walks the
//    v1 slices; each slice's rows are one contiguous block of the planogram,
//    fetched by a bulk copy (cp.async.bulk, no tensor map, no multicast) into
//    a ring of kPfdrStages slots two slices ahead of the computation;
//  * every warp transforms its own pair of rows (one complex sequence) with a
//    warp-synchronous radix-4/2 Stockham FFT whose sizes are compile-time
//    constants, and keeps the masked spectrum sums of its rows in registers;
//  * one CTA barrier per slice releases the slot to the next copy.
// Waits on the ring are bounded: a wait that gives up sets the device error
// word; the CTA then drains its copies in flight and returns without writing.
// ---------------------------------------------------------------------------
constexpr int kPfdrStages = 3;
constexpr int kPfdrWarps = kPfdrRows / 2;

// Work-buffer index of element i inside the FFT: bits 0-3 are XORed with 5
// times bits 4-5 (an involution on every block of 16).  The butterfly stores
// of the first two radix-4 stages go to indices 4j + c and 16 (j / 4) +
// 4c + j % 4; with the permutation each half warp's 16 stores (and every
// contiguous run of 16) hit 16 distinct bank pairs instead of 4.
__device__ __forceinline__ int fsw(int i) { return i ^ (((i >> 4) & 3) * 5); }

// Twiddles of the warp FFT in stage order: radix-4 stage s (Ns = 4^s) holds
// entries [k][r - 1] = tw[(r k N / (4 Ns)) mod N] at offset 4^s - 1, the
// radix-2 stage (when log2 N is odd) entries [k] = tw[k N / (2 Ns)] after
// them; fewer than N entries in all.  A half warp reads consecutive k, 24 or
// 8 bytes apart: distinct bank pairs.
template <int N>
__device__ void fill_stage_twiddles(float2* tws, const float2* __restrict__ tw, int tid, int nthreads)
{
    int off = 0, Ns = 1;
    for (; Ns * 4 <= N; off += 3 * Ns, Ns *= 4) {
        const int twstep = N / (Ns * 4);
        for (int e = tid; e < 3 * Ns; e += nthreads) {
            const int k = e / 3, r = e - 3 * k + 1;
            tws[off + e] = tw[(r * k * twstep) & (N - 1)];
        }
    }
    if (Ns < N) {
        const int twstep = N / (Ns * 2);
        for (int k = tid; k < Ns; k += nthreads) tws[off + k] = tw[(k * twstep) & (N - 1)];
    }
}

template <int N>
__device__ __forceinline__ void warp_fft(float2* a, float2* b, const float2* __restrict__ tws, float sign, int lane)
{
    // Stockham radix-4 stages, then one radix-2 stage when log2(N) is odd;
    // twiddles from fill_stage_twiddles (forward table, conjugated for the
    // inverse).  Input and result in a in natural order; the buffers
    // between stages are in fsw order.
    constexpr int n4 = []() { int n = 0; for (int m = 1; m * 4 <= N; m *= 4) n++; return n; }();
    constexpr bool has2 = (1 << (2 * n4)) < N;
    float2* src = a;
    float2* dst = b;
    int Ns = 1, off = 0;
#pragma unroll
    for (int s = 0; s < n4; s++) {
        constexpr int nbf = N / 4;
        const bool rsw = s > 0, wsw = has2 || s < n4 - 1;  // natural order at the ends
#pragma unroll
        for (int j = lane; j < nbf; j += 32) {
            const int k = j & (Ns - 1);
            float2 v[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int si = j + r * nbf;
                float2 x = src[rsw ? fsw(si) : si];
                if (r && k) {
                    float2 w = tws[off + 3 * k + r - 1];
                    w.y *= -sign;
                    x = cmul(x, w);
                }
                v[r] = x;
            }
            const float2 s02 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
            const float2 d02 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
            const float2 s13 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
            const float2 d13 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
            const float2 jd13 = make_float2(-sign * d13.y, sign * d13.x);
            const int idx = (j - k) * 4 + k;
            const float2 o[4] = {make_float2(s02.x + s13.x, s02.y + s13.y), make_float2(d02.x + jd13.x, d02.y + jd13.y),
                                 make_float2(s02.x - s13.x, s02.y - s13.y), make_float2(d02.x - jd13.x, d02.y - jd13.y)};
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int di = idx + c * Ns;
                dst[wsw ? fsw(di) : di] = o[c];
            }
        }
        __syncwarp();
        float2* t = src;
        src = dst;
        dst = t;
        off += 3 * Ns;
        Ns *= 4;
    }
    if (has2) {  // radix-2 stage: reads fsw order, writes natural order
        constexpr int nbf = N / 2;
#pragma unroll
        for (int j = lane; j < nbf; j += 32) {
            const int k = j & (Ns - 1);
            float2 x0 = src[fsw(j)], x1 = src[fsw(j + nbf)];
            if (k) {
                float2 w = tws[off + k];
                w.y *= -sign;
                x1 = cmul(x1, w);
            }
            const int idx = (j - k) * 2 + k;
            dst[idx] = make_float2(x0.x + x1.x, x0.y + x1.y);
            dst[idx + Ns] = make_float2(x0.x - x1.x, x0.y - x1.y);
        }
        __syncwarp();
        float2* t = src;
        src = dst;
        dst = t;
    }
    if (src != a) {
        for (int i = lane; i < N; i += 32) a[i] = src[i];
        __syncwarp();
    }
}

template <int NX>
__global__ void __launch_bounds__(kPfdrThreads) k_pfdr_stream(const PfdrArgs A, int* err, unsigned wlim)
{
    constexpr int NXH = NX / 2 + 1;
    constexpr int KPL = (NXH + 31) / 32;  // spectrum bins per lane
    extern __shared__ __align__(16) unsigned char smraw[];
    const int N_u0 = A.N_u0;
    const int stage_floats = kPfdrRows * N_u0;
    float* stage = reinterpret_cast<float*>(smraw);                                   // [S][rows][N_u0]
    float2* wbuf = reinterpret_cast<float2*>(stage + kPfdrStages * stage_floats);     // [warps][2][NX]
    float2* tw = wbuf + kPfdrWarps * 2 * NX;                                          // [NX]
    uint64_t* full = reinterpret_cast<uint64_t*>(tw + NX);                           // [S]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int iv0 = blockIdx.x;
    const int iu1_0 = blockIdx.y * kPfdrRows;
    const int nrows = min(kPfdrRows, A.N_u1 - iu1_0);
    const uint32_t bytes = uint32_t(nrows) * uint32_t(N_u0) * 4u;
    const size_t slab = size_t(A.N_v0) * A.N_u1 * N_u0;
    const float* base = A.g + (size_t(iv0) * A.N_u1 + iu1_0) * N_u0;
    const int nsl = A.N_v1;
    fill_stage_twiddles<NX>(tw, A.tw, tid, blockDim.x);
    if (tid == 0) {
        for (int q = 0; q < kPfdrStages; q++) mbar_init(&full[q], 1);
        fence_barrier_init();
    }
    __syncthreads();
    // load position q (the q-th slice in processing order) goes to slot q % S
    int issued = 0;  // meaningful in thread 0
    if (tid == 0)
        for (; issued < kPfdrStages && issued < nsl; issued++) {
            mbar_arrive_expect_tx(&full[issued], bytes);
            bulk_load(stage + issued * stage_floats, base + size_t(A.order[issued]) * slab, bytes, &full[issued]);
        }
    float2* a = wbuf + warp * 2 * NX;
    float2* b = a + NX;
    const int r0 = 2 * warp, r1 = 2 * warp + 1;  // rows of this warp's sequence
    float absU[KPL];
    float2 acc0[KPL], acc1[KPL];
#pragma unroll
    for (int m = 0; m < KPL; m++) {
        const int k = lane + 32 * m;
        absU[m] = k < NXH ? A.absU[k] : 0.0f;
        acc0[m] = make_float2(0.f, 0.f);
        acc1[m] = make_float2(0.f, 0.f);
    }
    bool dead = false;
    int gi = 0, q0 = 0;
    for (; gi < A.ngroups; gi++) {
        q0 = A.gfirst[gi];
        const int q1 = A.gfirst[gi + 1];
        for (int q = q0; q < q1 && !dead; q++)
            dead = !mbar_wait(&full[q % kPfdrStages], uint32_t((q / kPfdrStages) & 1), err, wlim);
        if (!dead) {
            // one or two slices: weights and staged rows hoisted out of the row loop
            const bool two = q1 - q0 > 1;
            const float w0 = A.row_w[A.order[q0] * A.N_v0 + iv0];
            const float w1 = two ? A.row_w[A.order[q0 + 1] * A.N_v0 + iv0] : 0.0f;
            const float* s0 = stage + (q0 % kPfdrStages) * stage_floats;
            const float* s1 = stage + ((q0 + 1) % kPfdrStages) * stage_floats;
            const int o0 = min(r0, nrows - 1) * N_u0, o1 = min(r1, nrows - 1) * N_u0;
            const bool v0 = r0 < nrows, v1 = r1 < nrows;
            for (int i = lane; i < NX; i += 32) {
                float re = 0.f, im = 0.f;
                if (i < N_u0) {
                    if (v0) re = s0[o0 + i] * w0;
                    if (v1) im = s0[o1 + i] * w0;
                    if (two) {
                        if (v0) re += s1[o0 + i] * w1;
                        if (v1) im += s1[o1 + i] * w1;
                    }
                }
                a[i] = make_float2(re, im);
            }
        }
        // the group's slots have been read: later slices may be copied in
        if (__syncthreads_or(dead)) break;
        if (tid == 0) {
            fence_proxy_async_smem();
            for (; issued < nsl && issued < q1 + kPfdrStages; issued++) {
                const int slot = issued % kPfdrStages;
                mbar_arrive_expect_tx(&full[slot], bytes);
                bulk_load(stage + slot * stage_floats, base + size_t(A.order[issued]) * slab, bytes, &full[slot]);
            }
        }
        __syncwarp();
        warp_fft<NX>(a, b, tw, -1.0f, lane);
        // split the two real spectra and accumulate the masked bins (the
        // group's slices share the mask)
        const int sl = A.order[q0];
        const bool cen = A.central[sl] != 0;
        const float thr = A.v1ap[sl];
#pragma unroll
        for (int m = 0; m < KPL; m++) {
            const int k = lane + 32 * m;
            if (k < NXH && (cen || absU[m] > thr)) {
                const float2 z = a[k];
                const float2 zc = a[k == 0 ? 0 : NX - k];
                acc0[m].x += 0.5f * (z.x + zc.x);
                acc0[m].y += 0.5f * (z.y - zc.y);
                acc1[m].x += 0.5f * (z.y + zc.y);
                acc1[m].y += -0.5f * (z.x - zc.x);
            }
        }
        __syncwarp();
    }
    if (gi < A.ngroups) {
        // a wait gave up: drain the copies in flight (load positions q0 ..
        // issued - 1, at most S of them; thread 0 tracks `issued`), write
        // nothing
        if (tid == 0)
            for (int q = q0; q < issued; q++) mbar_wait(&full[q % kPfdrStages], uint32_t((q / kPfdrStages) & 1), nullptr);
        return;
    }
    // normalise and pack the two rows into one inverse transform, A + iB:
    // the lane holding bin k writes bin k and its Hermitian image NX - k
#pragma unroll
    for (int m = 0; m < KPL; m++) {
        const int k = lane + 32 * m;
        if (k < NXH) {
            const float nr = A.norm[k];
            float2 x = make_float2(acc0[m].x * nr, acc0[m].y * nr), y = make_float2(acc1[m].x * nr, acc1[m].y * nr);
            const bool edge = k == 0 || 2 * k == NX;
            if (edge) {  // C2R ignores these imaginary parts
                x.y = 0.f;
                y.y = 0.f;
            }
            a[k] = make_float2(x.x - y.y, x.y + y.x);
            if (!edge) a[NX - k] = make_float2(x.x - (-y.y), (-x.y) + y.x);  // conjugates of both spectra
        }
    }
    __syncwarp();
    warp_fft<NX>(a, b, tw, 1.0f, lane);
    const float ow = A.out_w[iv0];
    for (int i = lane; i < N_u0; i += 32) {
        const float2 z = a[i];
        if (r0 < nrows) A.g_reb[(size_t(iv0) * A.N_u1 + iu1_0 + r0) * N_u0 + i] = z.x * ow;
        if (r1 < nrows) A.g_reb[(size_t(iv0) * A.N_u1 + iu1_0 + r1) * N_u0 + i] = z.y * ow;
    }
}

template <int NX>
cudaError_t launch_pfdr_stream(const PfdrArgs& A, cudaStream_t st)
{
    int* err = device_error_ptr();
    if (!err) return cudaErrorUnknown;
    const size_t smem = size_t(kPfdrStages) * kPfdrRows * A.N_u0 * 4 + sizeof(float2) * (size_t(kPfdrWarps) * 2 * NX + NX) +
                        sizeof(uint64_t) * kPfdrStages;
    cudaError_t e = cudaFuncSetAttribute(k_pfdr_stream<NX>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    dim3 grid(A.N_v0, ceil_div(A.N_u1, kPfdrRows));
    k_pfdr_stream<NX><<<grid, kPfdrThreads, smem, st>>>(A, err, wait_limit());
    note_launch();
    return cudaGetLastError();
}

// direct convolution of every row with the ramp kernel, times a per-view weight
constexpr int kRampRows = 8;
__global__ void __launch_bounds__(256)
k_ramp(float* __restrict__ g, int nrows, int N, int rows_per_view, const float* __restrict__ h,
       const float* __restrict__ view_w)
{
    extern __shared__ float rs[];
    float* hs = rs;              // 2N-1 taps, hs[N-1+s] = h(s)
    float* xs = hs + 2 * N - 1;  // kRampRows * N
    const int r0 = blockIdx.x * kRampRows;
    const int nr = min(kRampRows, nrows - r0);
    for (int i = threadIdx.x; i < 2 * N - 1; i += blockDim.x) hs[i] = h[i];
    for (int i = threadIdx.x; i < kRampRows * N; i += blockDim.x) {
        const int r = i / N;
        xs[i] = r < nr ? g[size_t(r0 + r) * N + (i - r * N)] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        float acc[kRampRows];
#pragma unroll
        for (int r = 0; r < kRampRows; r++) acc[r] = 0.f;
        for (int k = 0; k < N; k++) {
            const float hv = hs[N - 1 + i - k];
#pragma unroll
            for (int r = 0; r < kRampRows; r++) acc[r] = fmaf(xs[r * N + k], hv, acc[r]);
        }
        for (int r = 0; r < nr; r++) {
            const int row = r0 + r;
            g[size_t(row) * N + i] = acc[r] * view_w[row / rows_per_view];
        }
    }
}

// The same convolution with four adjacent outputs per thread: the taps of
// columns i0..i0+3 at input k are h[N-1+i0+j-k], a window that moves by one
// tap per k, so a thread loads one tap and eight row values per k for 32
// FMAs (the kernel above loads nine values for 8).  Per output the same
// fmaf chain over k in ascending order.  Block = 4 groups of 8 rows x 64
// column quads; rows of up to kRamp4MaxN floats.
constexpr int kRamp4Rows = 32;
constexpr int kRamp4MaxN = 1024;
__global__ void __launch_bounds__(256)
k_ramp4(float* __restrict__ g, int nrows, int N, int rows_per_view, const float* __restrict__ h,
        const float* __restrict__ view_w)
{
    extern __shared__ float rs[];
    float* hs = rs;                // 2N + 4 taps, hs[N-1+s] = h(s), zero past the last
    float* xs = hs + 2 * N + 4;    // kRamp4Rows * N
    const int r0 = blockIdx.x * kRamp4Rows;
    const int nr = min(kRamp4Rows, nrows - r0);
    for (int i = threadIdx.x; i < 2 * N + 4; i += blockDim.x) hs[i] = i < 2 * N - 1 ? h[i] : 0.0f;
    for (int i = threadIdx.x; i < kRamp4Rows * N; i += blockDim.x) {
        const int r = i / N;
        xs[i] = r < nr ? g[size_t(r0 + r) * N + (i - r * N)] : 0.0f;
    }
    __syncthreads();
    const int grp = threadIdx.x >> 6, q0 = threadIdx.x & 63;
    const float* xg = xs + grp * 8 * N;
    for (int q = q0; 4 * q < N; q += 64) {
        const int i0 = 4 * q;
        float acc[8][4];
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[r][j] = 0.f;
        float hw[4];  // hw[j] = h tap of column i0 + j at the current k
#pragma unroll
        for (int j = 0; j < 4; j++) hw[j] = hs[N - 1 + i0 + j];
        for (int k = 0; k < N; k++) {
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const float xv = xg[r * N + k];
#pragma unroll
                for (int j = 0; j < 4; j++) acc[r][j] = fmaf(xv, hw[j], acc[r][j]);
            }
            hw[3] = hw[2];
            hw[2] = hw[1];
            hw[1] = hw[0];
            hw[0] = k + 1 < N ? hs[N - 2 + i0 - k] : 0.0f;
        }
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int row = r0 + grp * 8 + r;
            if (grp * 8 + r >= nr) break;
            const float w = view_w[row / rows_per_view];
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (i0 + j < N) g[size_t(row) * N + i0 + j] = acc[r][j] * w;
        }
    }
}

// Device copies of the host-computed tables of a geometry, kept for later
// calls (per device, up to kTableCacheSize geometries, oldest dropped):
// building and uploading them per call from pageable memory kept the device
// idle for tens of microseconds before every PFDR launch.  An entry is one
// allocation holding every table at 256-byte aligned offsets; its upload is
// stream-ordered on the stream of the call that built it, and later calls
// on any stream wait for its event.
struct TableBlob {
    std::vector<unsigned char> bytes;
    size_t add(const void* src, size_t n)
    {
        const size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + n);
        std::memcpy(bytes.data() + off, src, n);
        return off;
    }
};

struct CachedTables {
    unsigned char* base = nullptr;
    cudaEvent_t ready = nullptr;
    unsigned long long last_use = 0;
    std::vector<size_t> off;  // offsets of the tables in the allocation
    std::vector<int> ints;    // host-side scalars the caller stores with them
};

constexpr size_t kTableCacheSize = 16;
std::mutex g_table_mu;
std::map<std::string, CachedTables> g_tables;
unsigned long long g_table_clock = 0;

// The cached tables under `key` (built by `make` on a miss: fills the blob
// and the scalars), the stream made to wait for their upload; null on a
// CUDA failure.  The caller holds g_table_mu until its launches that read
// the tables are enqueued (an eviction waits for the device to finish them).
template <class Make>
const CachedTables* cached_tables(const std::string& key0, cudaStream_t st, Make make)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const std::string key = key0 + std::string(reinterpret_cast<const char*>(&dev), sizeof(dev));
    auto it = g_tables.find(key);
    if (it == g_tables.end()) {
        if (g_tables.size() >= kTableCacheSize) {  // drop the least recently used
            auto old = g_tables.begin();
            for (auto jt = g_tables.begin(); jt != g_tables.end(); ++jt)
                if (jt->second.last_use < old->second.last_use) old = jt;
            cudaEventSynchronize(old->second.ready);  // its users' reads were enqueued after its upload
            cudaDeviceSynchronize();                   // and have finished
            cudaFree(old->second.base);
            cudaEventDestroy(old->second.ready);
            g_tables.erase(old);
        }
        CachedTables c;
        TableBlob blob;
        make(blob, c.off, c.ints);
        if (cudaMalloc(reinterpret_cast<void**>(&c.base), std::max<size_t>(blob.bytes.size(), 256)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        if (cudaMemcpyAsync(c.base, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.ready, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(c.ready, st) != cudaSuccess) {
            cudaFree(c.base);
            return nullptr;
        }
        it = g_tables.emplace(key, std::move(c)).first;
    } else if (cudaStreamWaitEvent(st, it->second.ready, 0) != cudaSuccess) {
        return nullptr;
    }
    it->second.last_use = ++g_table_clock;
    return &it->second;
}

// host float helpers that must not be contracted into fused multiply-adds
// (the reference computes these on the host with separate roundings)
__attribute__((noinline)) float fmul_h(float a, float b) { return a * b; }
__attribute__((noinline)) float fadd_h(float a, float b) { return a + b; }

}  // namespace

int pfdr(const petl_geom& G, const float* g, float* g_reb, cudaStream_t st)
{
    const int NX = petl_optimal_fft_size(G.N_u0);
    const FFTPlan plan = make_plan(NX);
    PETL_REQUIRE(plan.nstages > 0 && NX <= kMaxFFT, "PFDR: unsupported transform size");
    const int NXH = NX / 2 + 1;
    // the tables of the geometry (src/pfdr.cu:16-40, 78-124, 126-142,
    // 144-157), built on the host once per geometry
    auto make = [&](TableBlob& blob, std::vector<size_t>& off, std::vector<int>& ints) {
        const float T_U = float(1.0 / (NX * G.T_u0));
        const float aperture = float(1 / (2.0 * G.T_u1 * 2.0 * G.v_m0));
        std::vector<float> absU(NXH), v1ap(G.N_v1), row_w(size_t(G.N_v1) * G.N_v0), norm(NXH), out_w(G.N_v0);
        std::vector<unsigned char> central(G.N_v1);
        std::vector<float2> tw(NX);
        for (int i = 0; i < NXH; i++) {
            const float U = i < NX / 2 ? fmul_h(float(i), T_U) : fmul_h(float(i - NX), T_U);
            absU[i] = std::fabs(U);
        }
        std::vector<int> count(NXH, 0);
        for (int iv1 = 0; iv1 < G.N_v1; iv1++) {
            const float v1 = fadd_h(fmul_h(float(iv1), G.T_v1), G.v1_0);  // planogram::v1 on the host
            const float av = std::fabs(v1);
            central[iv1] = av <= fmul_h(0.5f, G.T_v1);
            v1ap[iv1] = fmul_h(av, aperture);
            for (int i = 0; i < NXH; i++)
                if (central[iv1] || absU[i] > v1ap[iv1]) count[i]++;
            for (int iv0 = 0; iv0 < G.N_v0; iv0++) {
                const float v0 = std::fmaf(G.T_v0, float(iv0), G.v0_0);  // device expression, contracted
                row_w[size_t(iv1) * G.N_v0 + iv0] = float(1.0 / std::sqrt(1.0 + double(v1) * v1 + double(v0) * v0));
            }
        }
        for (int i = 0; i < NXH; i++) norm[i] = float(1.0 / (double(NX) * ((i != 0 && count[i] > 0) ? count[i] : 1)));
        for (int iv0 = 0; iv0 < G.N_v0; iv0++) {
            const float v0 = std::fmaf(G.T_v0, float(iv0), G.v0_0);
            out_w[iv0] = float(std::sqrt(1.0 + double(v0) * v0));
        }
        const double PI = 3.14159265358979323846;
        for (int m = 0; m < NX; m++)
            tw[m] = make_float2(float(std::cos(-2.0 * PI * m / NX)), float(std::sin(-2.0 * PI * m / NX)));
        // processing order for the streamed kernel: slope iv1 with its mirror
        // N_v1 - 1 - iv1 when both have bit-identical masks (central flag and
        // threshold), else alone
        std::vector<int> order, gfirst;
        std::vector<char> done(G.N_v1, 0);
        for (int iv1 = 0; iv1 < G.N_v1; iv1++) {
            if (done[iv1]) continue;
            gfirst.push_back(int(order.size()));
            order.push_back(iv1);
            done[iv1] = 1;
            const int m = G.N_v1 - 1 - iv1;
            if (m != iv1 && !done[m] && central[m] == central[iv1] &&
                std::memcmp(&v1ap[m], &v1ap[iv1], sizeof(float)) == 0) {
                order.push_back(m);
                done[m] = 1;
            }
        }
        gfirst.push_back(int(order.size()));
        off = {blob.add(absU.data(), 4 * absU.size()), blob.add(v1ap.data(), 4 * v1ap.size()),
               blob.add(row_w.data(), 4 * row_w.size()), blob.add(norm.data(), 4 * norm.size()),
               blob.add(out_w.data(), 4 * out_w.size()), blob.add(central.data(), central.size()),
               blob.add(tw.data(), 8 * tw.size()), blob.add(order.data(), 4 * order.size()),
               blob.add(gfirst.data(), 4 * gfirst.size())};
        ints = {int(gfirst.size()) - 1};
    };
    std::lock_guard<std::mutex> lk(g_table_mu);
    const CachedTables* c = cached_tables(std::string("pfdr") + std::string(reinterpret_cast<const char*>(&G), sizeof G),
                                          st, make);
    if (!c) {
        set_error("PFDR: table upload failed");
        return int(cudaErrorMemoryAllocation);
    }
    PfdrArgs A{};
    A.g = g;
    A.g_reb = g_reb;
    A.N_v1 = G.N_v1; A.N_v0 = G.N_v0; A.N_u1 = G.N_u1; A.N_u0 = G.N_u0;
    A.NX = NX;
    A.plan = plan;
    A.absU = reinterpret_cast<const float*>(c->base + c->off[0]);
    A.v1ap = reinterpret_cast<const float*>(c->base + c->off[1]);
    A.row_w = reinterpret_cast<const float*>(c->base + c->off[2]);
    A.norm = reinterpret_cast<const float*>(c->base + c->off[3]);
    A.out_w = reinterpret_cast<const float*>(c->base + c->off[4]);
    A.central = c->base + c->off[5];
    A.tw = reinterpret_cast<const float2*>(c->base + c->off[6]);
    A.order = reinterpret_cast<const int*>(c->base + c->off[7]);
    A.gfirst = reinterpret_cast<const int*>(c->base + c->off[8]);
    A.ngroups = c->ints[0];
    // the streamed kernel: bulk copies need 16-byte aligned rows of slices
    const bool rows_ok = (G.N_u0 % 4) == 0 && (reinterpret_cast<uintptr_t>(g) & 15) == 0 && G.N_u0 <= NX &&
                         dispatch_mode() != 2;  // dispatch 2: the first-generation kernel
    cudaError_t e = cudaErrorNotSupported;
    if (rows_ok && NX == 128) e = launch_pfdr_stream<128>(A, st);
    else if (rows_ok && NX == 256) e = launch_pfdr_stream<256>(A, st);
    else if (rows_ok && NX == 512) e = launch_pfdr_stream<512>(A, st);
    else if (rows_ok && NX == 1024) e = launch_pfdr_stream<1024>(A, st);
    else {
        const size_t smem = sizeof(float2) * (size_t(2 * (kPfdrRows / 2) * NX) + size_t(kPfdrRows) * NXH + NX) +
                            sizeof(float) * NXH;
        e = cudaFuncSetAttribute(k_pfdr, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) {
            dim3 grid(G.N_v0, ceil_div(G.N_u1, kPfdrRows));
            k_pfdr<<<grid, kPfdrThreads, smem, st>>>(A);
            e = cudaGetLastError();
            note_launch();
        }
    }
    if (e != cudaSuccess) {
        set_error(std::string("PFDR: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

int ramp(const petl_geom& G, float* g_reb, int apply_weight, cudaStream_t st)
{
    const int N = G.N_u0;
    PETL_REQUIRE(N > 0 && N <= 4096, "ramp: unsupported row length");
    // h[s] = 1/(T pi (1/4 - s^2)) stored as float, as rampImpulseResponse
    auto make = [&](TableBlob& blob, std::vector<size_t>& off, std::vector<int>&) {
        std::vector<float> h(2 * N - 1);
        const double PI = 3.1415926535897932385;
        const float T = G.T_u0;
        for (int i = 0; i < 2 * N - 1; i++) {
            const float s = float(i - (N - 1));
            h[i] = float(1.0 / (T * PI * (0.25 - s * s)));
        }
        // inverse planogram weight per view (apply_planogram_weight(true))
        std::vector<float> vw(G.N_v0, 1.0f);
        if (apply_weight) {
            const float v1 = fadd_h(fmul_h(0.0f, G.T_v1), G.v1_0);
            for (int iv0 = 0; iv0 < G.N_v0; iv0++) {
                const float v0 = fadd_h(fmul_h(float(iv0), G.T_v0), G.v0_0);
                const float c = float(1.0 / std::sqrt(1.0 + double(v1) * v1 + double(v0) * v0));
                vw[iv0] = float(1.0 / c);
            }
        }
        off = {blob.add(h.data(), 4 * h.size()), blob.add(vw.data(), 4 * vw.size())};
    };
    std::lock_guard<std::mutex> lk(g_table_mu);
    const CachedTables* c = cached_tables(std::string(apply_weight ? "rampw" : "ramp") +
                                              std::string(reinterpret_cast<const char*>(&G), sizeof G),
                                          st, make);
    if (!c) {
        set_error("ramp: table upload failed");
        return int(cudaErrorMemoryAllocation);
    }
    const float* d_h = reinterpret_cast<const float*>(c->base + c->off[0]);
    const float* d_vw = reinterpret_cast<const float*>(c->base + c->off[1]);
    const int nrows = G.N_v0 * G.N_u1;
    // four columns per thread where the blocks of 32 rows still fill the
    // device twice over (at 4160 rows the 8-row blocks measured faster)
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    cudaError_t e;
    if (N <= kRamp4MaxN && nrows >= 2 * kRamp4Rows * sms) {
        const size_t smem = sizeof(float) * (size_t(2 * N + 4) + size_t(kRamp4Rows) * N);
        e = cudaFuncSetAttribute(k_ramp4, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) {
            k_ramp4<<<ceil_div(nrows, kRamp4Rows), 256, smem, st>>>(g_reb, nrows, N, G.N_u1, d_h, d_vw);
            e = cudaGetLastError();
            note_launch();
        }
    } else {
        const size_t smem = sizeof(float) * (size_t(2 * N - 1) + size_t(kRampRows) * N);
        e = cudaFuncSetAttribute(k_ramp, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) {
            k_ramp<<<ceil_div(nrows, kRampRows), 256, smem, st>>>(g_reb, nrows, N, G.N_u1, d_h, d_vw);
            e = cudaGetLastError();
            note_launch();
        }
    }
    if (e != cudaSuccess) {
        set_error(std::string("ramp: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl
