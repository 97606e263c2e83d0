// TMA-staged shear-warp projector and backprojectors (psi = 0, voxel pitch
// equal to the bin pitch).  They compute the operator of the first-generation
// kernels in projector_shear.cu (the shear-warp form of the reference
// footprint, src/projectors.cu:131-185 forward and :240-377 backward); only
// the staging and the register blocking differ.
//
// Forward, k_fwd_tma: one CTA per (view v0, 16 slopes v1, 32 rows u1, 64
// columns u0), 16 warps.  For each plane y that reaches the tile, one thread
// starts a TMA copy of the raw volume rows the tile needs (68 columns x nrb
// rows of plane y; whatever lies outside the volume arrives as zeros) up to
// four planes ahead of use.  The CTA interpolates the rows in x into shared
// memory once, then each warp applies the z interpolation of its 4 slopes
// for 8 rows from a single register window of 12 rows (the integer shifts of
// 4 consecutive slopes differ by at most 3 rows), two columns per lane.
//
// Backward, k_bwd_tma<ADJ>: one CTA per (8 planes y, 8 rows z, all columns),
// one column per lane, 16 warps.  For every (view v0, slope v1) whose rows
// reach the tile, one thread starts a TMA copy of the planogram rows the tile
// needs (N_u0 columns x brb rows) into a ring of up to 6 stages.  Each thread
// sums, for its 4 planes, the z-interpolated rows of every slope from one
// register window (the shifts of 4 consecutive planes differ by at most 2
// rows); after each view the x shift goes through shared memory into voxel
// accumulators held in registers.  Each voxel is owned by one CTA: no
// atomics, one write at the end.
//
// Both keep two warps' worth of independent FMA chains per scheduler with
// scalar FFMA: at this register budget (<= 128 per thread, 16 warps per SM)
// that issues at the full FP32 rate, which the packed f32x2 form does not.
//
// Every wait on a copy is bounded; a wait that gives up sets the device error
// word, and the CTA drains its copies in flight and stops without writing.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {
namespace shear {

namespace {

// ===========================================================================
// forward
// ===========================================================================
constexpr int FV = 4;              // slopes per warp
constexpr int FGV = 4;             // warps along v1
constexpr int FSL = FV * FGV;      // slopes per CTA
constexpr int FROWS = 16;          // rows per CTA
constexpr int FCOLS = 64;          // columns per CTA, two per lane
// staged raw columns: 64 + 1 tap + up to one 16-byte granule for alignment
template <class TF>
constexpr int fboxw() { return FCOLS + Store<TF>::kAlign; }
constexpr int FDMAX = 3;           // largest shift difference among a warp's slopes

struct FwdTmaArgs {
    petl_geom G;
    ViewRange vr;
    int n_colblk;  // ceil(N_u0 / 64)
    int nrb;       // staged rows per plane (32 + CTA shift spread + 1, bounded on the host)
    int nf;        // raw-row buffers in the copy ring
    int fstride;   // bytes per raw buffer
    int xstride;   // floats per interpolated buffer
    Tables T;
    int* err;
    unsigned wait_limit;  // bound of the waits on staged data (wait_limit(): kWaitLimit or 0)
};

struct FwdPlane {
    int cx;     // volume column of tile column 0 (before the x tap)
    int wlo;    // volume row of staged row 0
    int nr;     // staged rows used
    int dzmin;  // smallest z shift among the CTA's slopes
    float wx;   // x tap weight
};

// Plane geometry of a forward tile from the CTA's shared shift tables (x
// shifts of its view, z shifts of its slopes).  The z shift is monotone in
// v1, so the extreme shifts sit at the first and last slope.
__device__ __forceinline__ FwdPlane fwd_plane(const Shift* s_xt, const Shift* s_zt, int nsl, int NY, int col0,
                                              int row0, int y)
{
    const Shift xs = s_xt[y];
    const int da = s_zt[y].d, db = s_zt[(nsl - 1) * NY + y].d;
    FwdPlane p;
    p.dzmin = min(da, db);
    p.cx = col0 + xs.d;
    p.wx = xs.w;
    p.wlo = row0 + p.dzmin;
    p.nr = FROWS + (max(da, db) - p.dzmin) + 1;
    return p;
}

// z taps of one slope: all first-tap FMAs, then all second-tap FMAs (16
// independent chains per pass; per element the same order as one fused pass)
template <int O, int K>
__device__ __forceinline__ void fwd_taps(float2 (&acc)[K], const float2 (&W)[K + FDMAX + 1], float2 w0, float2 w1)
{
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = fma2(w0, W[k + O], acc[k]);
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = fma2(w1, W[k + O + 1], acc[k]);
}

// TF: volume storage, TG: planogram storage (float or bfloat16); the
// arithmetic is FP32 throughout.
template <int K, class TF, class TG>
__global__ void __launch_bounds__(32 * FGV * (FROWS / K), 2)
k_fwd_tma(const __grid_constant__ CUtensorMap fmap, TG* __restrict__ g, const TG* __restrict__ meas,
          const FwdTmaArgs A)
{
    constexpr int FBOXW = fboxw<TF>();
    constexpr int AL = Store<TF>::kAlign;
    constexpr int GR = FROWS / K;
    constexpr int NT = 32 * FGV * GR;
    constexpr int WN = K + FDMAX + 1;
    extern __shared__ __align__(128) unsigned char smem[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gv = warp % FGV, gr = warp / FGV;
    const int iv0 = A.vr.iv0_first + blockIdx.x * A.vr.iv0_step;
    const int v1a = A.vr.iv1_begin + blockIdx.y * FSL;
    const int v1b = min(v1a + FSL, A.vr.iv1_end) - 1;  // last slope of the CTA
    const int nsl = v1b - v1a + 1;
    const int rowblk = blockIdx.z / A.n_colblk, colblk = blockIdx.z % A.n_colblk;
    const int cta_row0 = rowblk * FROWS, col0 = colblk * FCOLS;
    const int jw = gv * FV;              // first slope of this warp, relative to v1a
    const int row0 = cta_row0 + gr * K;  // first row of this warp
    const int NY = G.numY, NZ = G.numZ, NX = G.numX;
    const int nf = A.nf;

    auto Fr = [&](int slot) {  // [nf][nrb][FBOXW] raw rows (TMA)
        return reinterpret_cast<TF*>(smem + size_t(slot) * A.fstride);
    };
    float* Xs = reinterpret_cast<float*>(smem + size_t(nf) * A.fstride);  // [4][nrb + 3][64] x-interpolated rows
    Shift* s_xt = reinterpret_cast<Shift*>(Xs + 4 * A.xstride);       // [NY] x shifts of view iv0
    Shift* s_zt = s_xt + NY;                                          // [nsl][NY] z shifts of the slopes
    uint64_t* bar = reinterpret_cast<uint64_t*>(s_zt + FSL * NY);     // [nf]
    int* s_n = reinterpret_cast<int*>(bar + nf);
    unsigned short* plist = reinterpret_cast<unsigned short*>(s_n + 2);  // live planes

    // a tile outside the visible bins of every slope stays zero
    const int2 ub0 = A.T.ub0[iv0];
    bool any_row = false;
    for (int v1 = v1a; v1 <= v1b; v1++) {
        const int2 u = A.T.ub1[v1];
        any_row |= !(cta_row0 > u.y || cta_row0 + FROWS - 1 < u.x);
    }
    const bool live = any_row && !(col0 > ub0.y || col0 + FCOLS - 1 < ub0.x);

    // slopes of this warp whose rows can be visible
    unsigned wmask = 0;
#pragma unroll
    for (int j = 0; j < FV; j++) {
        if (jw + j < nsl) {
            const int2 u = A.T.ub1[v1a + jw + j];
            if (!(row0 > u.y || row0 + K - 1 < u.x)) wmask |= 1u << j;
        }
    }

    float2 acc[FV][K];
#pragma unroll
    for (int j = 0; j < FV; j++)
#pragma unroll
        for (int k = 0; k < K; k++) acc[j][k] = make_float2(0.0f, 0.0f);

    if (live) {  // CTA-uniform
        // the shift tables this CTA reads, staged once (contiguous rows)
        for (int e = tid; e < NY; e += NT) s_xt[e] = A.T.xt[size_t(iv0) * NY + e];
        for (int e = tid; e < nsl * NY; e += NT) s_zt[e] = A.T.zt[size_t(v1a) * NY + e];
        __syncthreads();
        // planes whose staged window meets the volume, compacted in order
        if (warp == 0) {
            int n = 0;
            for (int yb = 0; yb < NY; yb += 32) {
                const int y = yb + lane;
                bool ok = false;
                if (y < NY) {
                    const FwdPlane p = fwd_plane(s_xt, s_zt, nsl, NY, col0, cta_row0, y);
                    ok = !(p.cx + FCOLS < 0 || p.cx >= NX || p.wlo + p.nr - 1 < 0 || p.wlo >= NZ);
                    if (ok && p.nr > A.nrb) {
                        atomicOr(A.err, kErrLayout);
                        ok = false;
                    }
                }
                const unsigned b = __ballot_sync(0xffffffffu, ok);
                if (ok) plist[n + __popc(b & ((1u << lane) - 1u))] = static_cast<unsigned short>(y);
                n += __popc(b);
            }
            if (lane == 0) {
                s_n[0] = n;
                for (int i = 0; i < nf; i++) mbar_init(&bar[i], 1);
                fence_barrier_init();
            }
        }
        __syncthreads();
        const int nlive = s_n[0];
        const uint32_t box_bytes = uint32_t(FBOXW) * uint32_t(A.nrb) * uint32_t(sizeof(TF));
        int issued = 0, islot = 0;  // thread 0 only: planes issued, ring slot of the next
        auto issue = [&](int li) {
            const int y = plist[li];
            const FwdPlane p = fwd_plane(s_xt, s_zt, nsl, NY, col0, cta_row0, y);
            mbar_arrive_expect_tx(&bar[islot], box_bytes);
            // x rounded down to a 16-byte granule: TMA needs 16-byte aligned starts
            tma_load_3d(Fr(islot), &fmap, &bar[islot], p.cx & ~(AL - 1), y, p.wlo);
            islot = (islot + 1 == nf) ? 0 : islot + 1;
        };
        if (tid == 0) {
            for (; issued < nf && issued < nlive; issued++) issue(issued);
        }

        // stage A: x interpolation of plane p's staged rows (raw slot rb) into
        // interpolated buffer xb, a row per warp, two adjacent columns per lane
        auto stage_a = [&](int rb, int xb, const FwdPlane& p) {
            const TF* F = Fr(rb) + (p.cx - (p.cx & ~(AL - 1))) + 2 * lane;
            float* X = Xs + xb * A.xstride + 2 * lane;
            const float w1 = p.wx, w0 = 1.0f - p.wx;
            for (int r = warp; r < p.nr; r += NT / 32) {
                const TF* fr = F + r * FBOXW;
                const float a = Store<TF>::ld(fr[0]), c = Store<TF>::ld(fr[1]), d = Store<TF>::ld(fr[2]);
                *reinterpret_cast<float2*>(X + r * FCOLS) = make_float2(fmaf(w1, c, w0 * a), fmaf(w1, d, w0 * c));
            }
        };
        // stage B: z interpolation of this warp's slopes on plane y from one window
        auto stage_b = [&](int xb, const FwdPlane& p, int y) {
            if (!wmask) return;  // warp-uniform
            Shift zs[FV];
            int base = 1 << 30;
#pragma unroll
            for (int j = 0; j < FV; j++) {
                zs[j] = Shift{0, 0.0f};
                if ((wmask >> j) & 1u) {
                    zs[j] = s_zt[(jw + j) * NY + y];
                    base = min(base, zs[j].d);
                }
            }
            const int xr0 = row0 - cta_row0 + base - p.dzmin;  // staged row of window row 0
            const int iz0 = p.wlo + xr0;                        // its volume row
            if (base < p.dzmin) {  // the shifts are monotone in v1; never read before the buffer
                atomicOr(A.err, kErrLayout);
                return;
            }
            if (iz0 + WN - 1 < 0 || iz0 >= NZ) return;  // window outside the volume: zeros
            const float* Xr = Xs + xb * A.xstride + xr0 * FCOLS + 2 * lane;
            float2 W[WN];
#pragma unroll
            for (int i = 0; i < WN; i++) W[i] = *reinterpret_cast<const float2*>(Xr + i * FCOLS);
#pragma unroll
            for (int j = 0; j < FV; j++) {
                if (!((wmask >> j) & 1u)) continue;
                const float2 w1 = dup(zs[j].w), w0 = dup(1.0f - zs[j].w);
                switch (zs[j].d - base) {
                    case 0: fwd_taps<0, K>(acc[j], W, w0, w1); break;
                    case 1: fwd_taps<1, K>(acc[j], W, w0, w1); break;
                    case 2: fwd_taps<2, K>(acc[j], W, w0, w1); break;
                    case 3: fwd_taps<3, K>(acc[j], W, w0, w1); break;
                    default: atomicOr(A.err, kErrLayout);
                }
            }
        };

        // two planes per CTA barrier: stage A of both, one barrier, stage B of
        // both; pairs alternate between two pairs of interpolated buffers
        bool dead = false;
        int li = 0, b = 0;   // first plane of the pair, its ring slot
        uint32_t phase = 0;  // parity of that slot's current use
        for (; li < nlive; li += 2) {
            const bool two = li + 1 < nlive;
            const int xq = 2 * ((li >> 1) & 1);
            int b1 = b + 1;
            uint32_t phase1 = phase;
            if (b1 == nf) {
                b1 = 0;
                phase1 ^= 1u;
            }
            const int y0 = plist[li], y1 = two ? plist[li + 1] : y0;
            const FwdPlane p0 = fwd_plane(s_xt, s_zt, nsl, NY, col0, cta_row0, y0);
            const FwdPlane p1 = fwd_plane(s_xt, s_zt, nsl, NY, col0, cta_row0, y1);
            if (!dead) dead = !mbar_wait(&bar[b], phase, A.err, A.wait_limit);
            stage_a(b, xq, p0);
            if (two) {
                if (!dead) dead = !mbar_wait(&bar[b1], phase1, A.err, A.wait_limit);
                stage_a(b1, xq + 1, p1);
            }
            if (__syncthreads_or(dead)) break;
            // every thread is done with the pair's raw slots: stage the planes nf later
            if (tid == 0) {
                fence_proxy_async_smem();
                for (int n = 0; n < (two ? 2 : 1) && issued < nlive; n++, issued++) issue(issued);
            }
            stage_b(xq, p0, y0);
            if (two) stage_b(xq + 1, p1, y1);
            b = b1;
            phase = phase1;
            if (two && ++b == nf) {
                b = 0;
                phase ^= 1u;
            }
        }
        if (li < nlive) {
            // a wait gave up: drain the copies still in flight, write nothing
            if (tid == 0)
                for (int q = li; q < issued; q++) mbar_wait(&bar[q % nf], uint32_t((q / nf) & 1), nullptr);
            return;
        }
    }

    // epilogue: scale, ray masks, optional MLEM ratio
    const int colA = col0 + 2 * lane;
    const bool pairs = (G.N_u0 & 1) == 0;  // float2 accesses stay 8-byte aligned
#pragma unroll
    for (int j = 0; j < FV; j++) {
        const int v1 = v1a + jw + j;
        if (jw + j >= nsl) continue;
        const float S = A.T.S[size_t(v1) * G.N_v0 + iv0];
        const int2 u1r = A.T.ub1[v1];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int iu1 = row0 + k;
            if (iu1 >= G.N_u1) break;
            const bool rv = iu1 >= u1r.x && iu1 <= u1r.y;
            const size_t o = ((size_t(v1) * G.N_v0 + iv0) * G.N_u1 + iu1) * G.N_u0 + colA;
            const bool v0ok = rv && colA >= ub0.x && colA <= ub0.y;
            const bool v1ok = rv && colA + 1 >= ub0.x && colA + 1 <= ub0.y;
            float2 val = make_float2(v0ok ? acc[j][k].x * S : 0.0f, v1ok ? acc[j][k].y * S : 0.0f);
            if (pairs && colA + 1 < G.N_u0) {
                if (meas) {
                    const float2 m = Store<TG>::ld2(meas + o);
                    val = make_float2(ratio_rule(m.x, val.x), ratio_rule(m.y, val.y));
                }
                Store<TG>::st2(g + o, val);
            } else {
                if (colA < G.N_u0) g[o] = Store<TG>::st(meas ? ratio_rule(Store<TG>::ld(meas[o]), val.x) : val.x);
                if (colA + 1 < G.N_u0)
                    g[o + 1] = Store<TG>::st(meas ? ratio_rule(Store<TG>::ld(meas[o + 1]), val.y) : val.y);
            }
        }
    }
}

// ===========================================================================
// backward
// ===========================================================================
constexpr int BK = 8;               // z rows per CTA
constexpr int BPT = 4;              // planes per thread
constexpr int BPG = 2;              // plane groups (at most)
constexpr int BNP = BPT * BPG;      // planes per CTA (at most)
constexpr int BDW = 2;              // largest shift difference among a thread's planes
constexpr int BWN = BK + BDW + 1;   // register window rows
constexpr int BNSMAX = 6;          // copy ring stages at most
constexpr int BV1CAP = 96;          // slopes held in the per-CTA tables

// Window offsets of a plane group's 4 planes when all are fully visible and
// their shifts differ by at most one row (monotone in y, the common case):
// one straight-line block of FMAs per stage.  Any other group takes the
// per-plane path (kPatGeneric).
constexpr int kNumPat = 7;
constexpr int kPatGeneric = 15;
__host__ __device__ constexpr int pat_offsets(int pid)
{
    // o0 | o1 << 2 | o2 << 4 | o3 << 6
    return pid == 0 ? 0x00 : pid == 1 ? 0x40 : pid == 2 ? 0x50 : pid == 3 ? 0x54
         : pid == 4 ? 0x01 : pid == 5 ? 0x05 : 0x15;
}

struct BwdTmaArgs {
    petl_geom G;
    ViewRange vr;
    int ncw;      // column warps per plane group (32 columns each)
    int brb;      // staged rows per view (>= BWN + CTA shift spread, bounded on the host)
    int sstride;  // bytes per ring stage
    int ns;       // ring stages
    int max_views;  // views the x-shift table holds
    int accumulate;
    float scale;
    Tables T;
    int* err;
    unsigned wait_limit;  // bound of the waits on staged data (wait_limit(): kWaitLimit or 0)
};

// z taps of one plane: Z[k] += w1 g[row k of tap 1] + w0 g[row k of tap 0],
// window row O + k holding tap 1 and O + k + 1 tap 0.  MASK applies per-row
// 0/1 factors: vm (window rows that hold visible bins, the adjoint's bin mask)
// and om (output rows inside the reference backprojector's voxel test).
template <int O, bool MASK>
__device__ __forceinline__ void bwd_taps(float (&Z)[BK], const float (&W)[BWN], float w0, float w1, uint32_t vm,
                                         uint32_t om)
{
    if (MASK) {
        // masked taps read zero instead of the window value (rows outside the
        // view are not copied and may hold any bit pattern, which a zero
        // weight would not cancel)
#pragma unroll
        for (int k = 0; k < BK; k++) {
            const float b = ((vm >> (O + k + 1)) & (om >> k) & 1u) ? W[O + k + 1] : 0.0f;
            const float a = ((vm >> (O + k)) & (om >> k) & 1u) ? W[O + k] : 0.0f;
            Z[k] = fmaf(w1, a, fmaf(w0, b, Z[k]));
        }
    } else {
        // all tap-0 FMAs, then all tap-1 FMAs: independent chains back to back
#pragma unroll
        for (int k = 0; k < BK; k++) Z[k] = fmaf(w0, W[O + k + 1], Z[k]);
#pragma unroll
        for (int k = 0; k < BK; k++) Z[k] = fmaf(w1, W[O + k], Z[k]);
    }
}

// z taps of a fully visible plane group with compile-time window offsets
template <int PID>
__device__ __forceinline__ void bwd_taps4(float (&Z)[BPT][BK], const float (&W)[BWN], float4 wa, float4 wb)
{
    constexpr int o = pat_offsets(PID);
    bwd_taps<(o >> 0) & 3, false>(Z[0], W, wa.x, wa.y, 0u, 0u);
    bwd_taps<(o >> 2) & 3, false>(Z[1], W, wa.z, wa.w, 0u, 0u);
    bwd_taps<(o >> 4) & 3, false>(Z[2], W, wb.x, wb.y, 0u, 0u);
    bwd_taps<(o >> 6) & 3, false>(Z[3], W, wb.z, wb.w, 0u, 0u);
}

// PITCH > 0: the planogram row pitch N_u0 as a compile-time constant (shared
// memory offsets become immediates); 0: read it from the geometry.
// TG: planogram storage, TF: volume storage (float or bfloat16); FP32
// arithmetic throughout.
// BULK: the planogram rows arrive by plain bulk copies (cp.async.bulk) of
// whole row pairs instead of a tensor map, which lifts the tensor map's rule
// that rows be multiples of 16 bytes and its 256-element box (N_u0 need only
// be even); rows outside the view are not copied and are masked instead.
// PG: plane groups per CTA (2, or 1 when N_u0 or numX exceeds 256).
template <bool ADJ, int PITCH, class TG, class TF, bool BULK, int PG>
__global__ void __launch_bounds__(512, 1)
k_bwd_tma(const __grid_constant__ CUtensorMap gmap, const TG* __restrict__ gsrc, TF* __restrict__ f,
          const BwdTmaArgs A)
{
    constexpr int NP = BPT * PG;  // planes per CTA
    extern __shared__ __align__(128) unsigned char smem[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    const int cw = warp % A.ncw, pg = warp / A.ncw;
    const int p0 = blockIdx.x * NP;  // first plane of the CTA
    const int r0 = blockIdx.y * BK;   // first z row of the CTA
    const int u = cw * 32 + lane;     // this thread's column (planogram u0 and voxel x)
    const int NY = G.numY, NX = G.numX, NZ = G.numZ, NU1 = G.N_u1;
    const int NU0 = PITCH > 0 ? PITCH : G.N_u0;
    const int n_v0 = A.vr.n_v0(G.N_v0);

    const int ns = A.ns;
    auto ring = [&](int slot) {  // [ns][brb][NU0] planogram rows (TMA)
        return reinterpret_cast<TG*>(smem + size_t(slot) * A.sstride);
    };
    float* Zs = reinterpret_cast<float*>(smem + size_t(ns) * A.sstride);  // [NP][BK][NU0]
    float2* Wt = reinterpret_cast<float2*>(Zs + NP * BK * NU0);          // [BV1CAP][NP]
    float* s_w = reinterpret_cast<float*>(Wt + BV1CAP * NP);             // [BV1CAP][NP]
    Shift* s_xs = reinterpret_cast<Shift*>(s_w + BV1CAP * NP);           // [n_v0][NP] x shifts of the planes
    int* s_v1 = reinterpret_cast<int*>(s_xs + A.max_views * NP);         // [BV1CAP]
    int* s_grow = s_v1 + BV1CAP;                                          // [BV1CAP]
    uint32_t* s_code = reinterpret_cast<uint32_t*>(s_grow + BV1CAP);      // [BV1CAP]
    uint32_t* s_wb = s_code + BV1CAP;                                     // [BV1CAP]
    uint32_t* s_mask = s_wb + BV1CAP;                                     // [BV1CAP][PG]
    uint32_t* s_vmask = s_mask + BV1CAP * PG;                            // [BV1CAP][PG]
    uint32_t* s_pat = s_vmask + BV1CAP * PG;                             // [BV1CAP]
    uint64_t* full = reinterpret_cast<uint64_t*>(s_pat + BV1CAP);         // [ns]
    uint64_t* empty = full + BNSMAX;                                      // [ns]
    int* s_n = reinterpret_cast<int*>(empty + BNSMAX);
    volatile int* s_abort = s_n + 1;  // a consumer gave up a wait: start no further copies
    int* s_round = s_n + 2;                                               // [ns]

    // ---- per-CTA slope tables (warp 0): for every slope whose rows reach the
    // tile, the staged g row, per plane the window offset and mode (0 none,
    // 1 full, 2 masked rows), per plane group the window base row.
    if (warp == 0) {
        int n = 0;
        for (int vb = A.vr.iv1_begin; vb < A.vr.iv1_end; vb += 32) {
            const int v1 = vb + lane;
            bool ok = false;
            uint32_t code = 0, wbs = 0, pats = 0;
            uint32_t msk[PG], vmsk[PG];
            int grow = 0;
            float wz[NP];
#pragma unroll
            for (int q = 0; q < PG; q++) msk[q] = vmsk[q] = 0xffffffffu;
            if (v1 < A.vr.iv1_end) {
                int dz[NP];
                int dmin = 1 << 30, dmax = -(1 << 30);
#pragma unroll
                for (int p = 0; p < NP; p++) {
                    const int y = min(p0 + p, NY - 1);
                    const Shift zs = A.T.zt[size_t(v1) * NY + y];
                    dz[p] = zs.d;
                    wz[p] = zs.w;
                    if (p0 + p < NY) {
                        dmin = min(dmin, zs.d);
                        dmax = max(dmax, zs.d);
                    }
                }
                grow = r0 - dmax - 1;
                const int2 ub1 = A.T.ub1[v1];
                int mode[NP];
#pragma unroll
                for (int p = 0; p < NP; p++) {
                    mode[p] = 0;
                    if (p0 + p >= NY) continue;
                    const int lo = r0 - dz[p] - 1, hi = r0 + BK - 1 - dz[p];  // g rows touched
                    if (hi < 0 || lo >= NU1) continue;
                    if (ADJ) {
                        if (hi < ub1.x || lo > ub1.y) continue;
                        mode[p] = (lo >= ub1.x && hi <= ub1.y) ? 1 : 2;
                    } else {
                        const int2 zv = A.T.zvis[size_t(v1) * NY + p0 + p];
                        if (r0 + BK - 1 < zv.x || r0 > zv.y) continue;
                        mode[p] = (r0 >= zv.x && r0 + BK - 1 <= zv.y) ? 1 : 2;
                    }
                    // bulk copies leave rows outside the view unwritten: mask them
                    if (BULK && mode[p] == 1 && (lo < 0 || hi >= NU1)) mode[p] = 2;
                }
                bool bad = dmax - dmin > A.brb - BWN;
#pragma unroll
                for (int q = 0; q < PG; q++) {
                    int wb = 1 << 30;
#pragma unroll
                    for (int t = 0; t < BPT; t++)
                        if (mode[q * BPT + t]) wb = min(wb, dmax - dz[q * BPT + t]);
                    if (wb == (1 << 30)) wb = 0;
#pragma unroll
                    for (int t = 0; t < BPT; t++) {
                        const int p = q * BPT + t;
                        if (!mode[p]) continue;
                        const int o = dmax - dz[p] - wb;
                        if (o > BDW) bad = true;
                        code |= uint32_t(mode[p] | (min(o, 3) << 2)) << (4 * p);
                        ok = true;
                    }
                    wbs |= uint32_t(wb) << (8 * q);
                    if (BULK) {
                        uint32_t vr = 0;  // window rows inside the view
                        for (int i = 0; i < BWN; i++)
                            if (grow + wb + i >= 0 && grow + wb + i < NU1) vr |= 1u << i;
                        vmsk[q] = vr;
                    }
                    // straight-line pattern of the group, if it has one
                    int pid = kPatGeneric;
                    {
                        bool allfull = true;
                        int offs = 0;
#pragma unroll
                        for (int t = 0; t < BPT; t++) {
                            const int p = q * BPT + t;
                            const int o = dmax - dz[p] - wb;
                            allfull = allfull && mode[p] == 1 && o <= 1;
                            offs |= (o & 3) << (2 * t);
                        }
                        if (allfull)
                            for (int c = 0; c < kNumPat; c++)
                                if (pat_offsets(c) == offs) pid = c;
                    }
                    pats |= uint32_t(pid) << (4 * q);
                    // row masks for planes at the edge of the visible range:
                    // adjoint, window rows holding visible bins of the group;
                    // reference, per plane the output rows passing the voxel test
                    if (ADJ) {
                        uint32_t vm = 0;
                        for (int i = 0; i < BWN; i++)
                            if (grow + wb + i >= ub1.x && grow + wb + i <= ub1.y) vm |= 1u << i;
                        msk[q] = vm & vmsk[q];
                    } else {
                        uint32_t om = 0;
#pragma unroll
                        for (int t = 0; t < BPT; t++) {
                            const int p = q * BPT + t;
                            if (mode[p] != 2) continue;
                            const int2 zv = A.T.zvis[size_t(v1) * NY + p0 + p];
                            for (int k = 0; k < BK; k++)
                                if (r0 + k >= zv.x && r0 + k <= zv.y) om |= 1u << (8 * t + k);
                        }
                        msk[q] = om;
                    }
                }
                if (ok && bad) {
                    atomicOr(A.err, kErrLayout);
                    ok = false;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int idx = n + __popc(bal & ((1u << lane) - 1u));
                if (idx < BV1CAP) {
                    s_v1[idx] = v1;
                    s_grow[idx] = grow;
                    s_code[idx] = code;
                    // bits 24..: the row of the copied pair block where row grow sits
                    s_wb[idx] = wbs | (BULK ? uint32_t(grow & 1) << 24 : 0u);
                    s_pat[idx] = pats;
#pragma unroll
                    for (int q = 0; q < PG; q++) s_vmask[idx * PG + q] = vmsk[q];
#pragma unroll
                    for (int q = 0; q < PG; q++) s_mask[idx * PG + q] = msk[q];
#pragma unroll
                    for (int p = 0; p < NP; p++) s_w[idx * NP + p] = wz[p];
                }
            }
            n += __popc(bal);
        }
        if (lane == 0) {
            if (n > BV1CAP) {  // the host caps the slope range; never index past the tables
                atomicOr(A.err, kErrLayout);
                n = BV1CAP;
            }
            s_n[0] = n;
            *s_abort = 0;
            for (int s = 0; s < ns; s++) {
                mbar_init(&full[s], 1);
                mbar_init(&empty[s], nwarps);
                s_round[s] = -1;
            }
            fence_barrier_init();
        }
    }
    __syncthreads();
    const int nlive = s_n[0];
    const long long total = (long long)n_v0 * nlive;

    // weights of view v0: (S w0, S w1) per live slope and plane.  The global
    // loads of S for the next view are issued at the start of a view
    // (load_S) and stored after its stages (store_w), so their latency hides
    // behind the view's work; at most kWPT elements per thread.
    constexpr int kWPT = (BV1CAP * NP + 511) / 512;
    float s_pre[kWPT];
    auto load_S = [&](int v0) {
#pragma unroll
        for (int i = 0; i < kWPT; i++) {
            const int e = tid + i * int(blockDim.x);
            s_pre[i] = e < nlive * NP ? __ldg(&A.T.S[size_t(s_v1[e / NP]) * G.N_v0 + v0]) : 0.0f;
        }
    };
    auto store_w = [&]() {
#pragma unroll
        for (int i = 0; i < kWPT; i++) {
            const int e = tid + i * int(blockDim.x);
            if (e < nlive * NP) {
                const float S = s_pre[i], w = s_w[e];
                Wt[e] = make_float2(S * (1.0f - w), S * w);
            }
        }
    };
    // x shifts of the CTA's planes for every view, staged once
    for (int e = tid; e < n_v0 * NP; e += blockDim.x) {
        const int iv = e / NP, p = e % NP;
        const int y = min(p0 + p, NY - 1);
        s_xs[e] = A.T.xt[size_t(A.vr.iv0_first + iv * A.vr.iv0_step) * NY + y];
    }
    const uint32_t box_bytes = uint32_t(NU0) * uint32_t(A.brb) * uint32_t(sizeof(TG));
    // Stage j is started by lane 0 of warp j % nwarps once every warp has
    // released its ring slot (the consumption of stage j - ns): the producer
    // work and its waits rotate over the warps instead of slowing one warp,
    // which would hold every other warp back through the empty barriers.
    // s_round[slot] records the round of the copy last started in a slot (for
    // draining after a failed wait).
    bool dead = false;
    const int ntot = int(total);
    auto issue = [&](int j) {
        const int slot = j % ns, round = j / ns;
        const int li = j % nlive;
        const int v0 = A.vr.iv0_first + (j / nlive) * A.vr.iv0_step;
        if (round > 0 && !mbar_wait(&empty[slot], uint32_t((round - 1) & 1), A.err, A.wait_limit)) return false;
        // a warp that gave up released its slot without its copy confirmed:
        // no copy may start into a slot after that
        if (*s_abort) return false;
        fence_proxy_async_smem();
        if constexpr (BULK) {
            // row pairs [rp0, rp0 + nrows) of view (v1, v0), the part inside
            // the view; even rows start 16-byte aligned (N_u0 and N_u1 even)
            const int gr = s_grow[li], rp0 = gr & ~1;
            const int nrows = (gr - rp0 + A.brb + 1) & ~1;
            const int ra = max(rp0, 0), rb = min(rp0 + nrows, NU1);
            const uint32_t bytes = rb > ra ? uint32_t(rb - ra) * uint32_t(NU0) * uint32_t(sizeof(TG)) : 0u;
            mbar_arrive_expect_tx(&full[slot], bytes);
            if (bytes) {
                const TG* src = gsrc + ((size_t(s_v1[li]) * G.N_v0 + v0) * NU1 + ra) * NU0;
                bulk_load(ring(slot) + (ra - rp0) * NU0, src, bytes, &full[slot]);
            }
        } else {
            mbar_arrive_expect_tx(&full[slot], box_bytes);
            tma_load_4d(ring(slot), &gmap, &full[slot], 0, s_grow[li], v0, s_v1[li]);
        }
        s_round[slot] = round;
        return true;
    };
    if (tid == 0)
        for (int j = 0; j < ns - 1 && j < ntot; j++) issue(j);
    // the next stage this warp starts: the first j >= ns - 1 with j % nwarps == warp
    int my_next = warp + nwarps * ((ns - 1 - warp + nwarps - 1) / nwarps);
    if (my_next < ns - 1) my_next += nwarps;
    if (n_v0 > 0) {
        load_S(A.vr.iv0_first);
        store_w();
    }
    __syncthreads();

    float Fv[BPT][BK];  // voxel accumulators (unscaled)
    float Z[BPT][BK];   // z-interpolated sums of the current view
#pragma unroll
    for (int q = 0; q < BPT; q++)
#pragma unroll
        for (int k = 0; k < BK; k++) {
            Fv[q][k] = 0.0f;
            Z[q][k] = 0.0f;
        }

    bool aborted = false;
    const bool ucol = u < NU0;
    long long it = 0;
    int c_slot = 0;         // ring slot of stage it
    uint32_t c_phase = 0;   // parity of that slot's current use
    for (int iv = 0; iv < n_v0 && !aborted; iv++) {
        const int v0 = A.vr.iv0_first + iv * A.vr.iv0_step;
        if (iv + 1 < n_v0) load_S(v0 + A.vr.iv0_step);
        for (int li = 0; li < nlive; li++, it++) {
            if (it + ns - 1 == my_next) {
                if (lane == 0 && !dead && my_next < ntot && !issue(my_next)) dead = true;
                my_next += nwarps;
            }
            const int s = c_slot;
            if (!dead) dead = !mbar_wait(&full[s], c_phase, A.err, A.wait_limit);
            if (dead) *s_abort = 1;  // before this warp releases the slot
            const uint32_t code = s_code[li] >> (16 * pg);  // this group's 4 planes
            const uint32_t pat = (s_pat[li] >> (4 * pg)) & 15u;
            if (dead) {
                // the slot's data may not have arrived: nothing is read
            } else if (ucol && pat != uint32_t(kPatGeneric)) {
                const uint32_t wbw = s_wb[li];
                const int wb = int((wbw >> (8 * pg)) & 0xff) + (BULK ? int(wbw >> 24) : 0);
                const TG* Gs = ring(s) + wb * NU0 + u;
                float W[BWN];
#pragma unroll
                for (int i = 0; i < BWN; i++) W[i] = Store<TG>::ld(Gs[i * NU0]);
                const float4* W4 = reinterpret_cast<const float4*>(Wt + li * NP + pg * BPT);
                const float4 wa = W4[0], wb4 = W4[1];
                switch (pat) {
                    case 0: bwd_taps4<0>(Z, W, wa, wb4); break;
                    case 1: bwd_taps4<1>(Z, W, wa, wb4); break;
                    case 2: bwd_taps4<2>(Z, W, wa, wb4); break;
                    case 3: bwd_taps4<3>(Z, W, wa, wb4); break;
                    case 4: bwd_taps4<4>(Z, W, wa, wb4); break;
                    case 5: bwd_taps4<5>(Z, W, wa, wb4); break;
                    default: bwd_taps4<6>(Z, W, wa, wb4); break;
                }
            } else if (ucol && (code & 0x3333u)) {
                const uint32_t wbw = s_wb[li];
                const int wb = int((wbw >> (8 * pg)) & 0xff) + (BULK ? int(wbw >> 24) : 0);
                const TG* Gs = ring(s) + wb * NU0 + u;
                float W[BWN];
#pragma unroll
                for (int i = 0; i < BWN; i++) W[i] = Store<TG>::ld(Gs[i * NU0]);
                const float2* Wl = Wt + li * NP + pg * BPT;
#pragma unroll
                for (int q = 0; q < BPT; q++) {
                    const uint32_t c = (code >> (4 * q)) & 15u;
                    if (!(c & 3u)) continue;
                    const float2 w = Wl[q];
                    const float w0 = w.x, w1 = w.y;
                    const int o = int(c >> 2);
                    if ((c & 3u) == 1u) {
                        switch (o) {
                            case 0: bwd_taps<0, false>(Z[q], W, w0, w1, 0u, 0u); break;
                            case 1: bwd_taps<1, false>(Z[q], W, w0, w1, 0u, 0u); break;
                            default: bwd_taps<2, false>(Z[q], W, w0, w1, 0u, 0u); break;
                        }
                    } else {
                        // rows at the edge of the visible range: per-row masks
                        const uint32_t m = s_mask[li * PG + pg];
                        const uint32_t vm = ADJ ? m : (BULK ? s_vmask[li * PG + pg] : 0xffffffffu);
                        const uint32_t om = ADJ ? 0xffffffffu : (m >> (8 * q)) & 0xffu;
                        switch (o) {
                            case 0: bwd_taps<0, true>(Z[q], W, w0, w1, vm, om); break;
                            case 1: bwd_taps<1, true>(Z[q], W, w0, w1, vm, om); break;
                            default: bwd_taps<2, true>(Z[q], W, w0, w1, vm, om); break;
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            if (++c_slot == ns) {
                c_slot = 0;
                c_phase ^= 1u;
            }
        }
        // ---- x shift of view v0 into the voxel accumulators
        {
            int2 u0r = make_int2(0, NU0 - 1);
            if (ADJ) u0r = A.T.ub0[v0];
#pragma unroll
            for (int q = 0; q < BPT; q++)
#pragma unroll
                for (int k = 0; k < BK; k++) {
                    if (ucol) {
                        const bool vis = !ADJ || (u >= u0r.x && u <= u0r.y);
                        Zs[((pg * BPT + q) * BK + k) * NU0 + u] = vis ? Z[q][k] : 0.0f;
                    }
                    Z[q][k] = 0.0f;
                }
        }
        if (__syncthreads_or(dead)) {
            aborted = true;
            break;
        }
#pragma unroll
        for (int q = 0; q < BPT; q++) {
            const int y = p0 + pg * BPT + q;
            if (y >= NY) continue;
            const Shift xs = s_xs[iv * NP + pg * BPT + q];
            const float wx1 = xs.w, wx0 = 1.0f - xs.w;
            const int j0 = u - xs.d;  // Z column of tap 0 for voxel column u
#pragma unroll
            for (int k = 0; k < BK; k++) {
                const float* zr = Zs + ((pg * BPT + q) * BK + k) * NU0;
                const float zm = (j0 - 1 >= 0 && j0 - 1 < NU0) ? zr[j0 - 1] : 0.0f;
                const float z0 = (j0 >= 0 && j0 < NU0) ? zr[j0] : 0.0f;
                Fv[q][k] += fmaf(wx1, zm, wx0 * z0);
            }
        }
        if (iv + 1 < n_v0) store_w();
        __syncthreads();
    }
    if (aborted) {
        // a wait gave up: drain the copies still in flight, write nothing
        __syncthreads();
        if (tid == 0)
            for (int slot = 0; slot < ns; slot++)
                if (s_round[slot] >= 0) mbar_wait(&full[slot], uint32_t(s_round[slot] & 1), nullptr);
        return;
    }

    // ---- the owned voxels, written once
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int y = p0 + pg * BPT + q;
        if (y >= NY) continue;
#pragma unroll
        for (int k = 0; k < BK; k++) {
            const int z = r0 + k;
            if (z >= NZ) break;
            TF* fr = f + (size_t(z) * NY + y) * NX;
            if (u < NX)
                fr[u] = Store<TF>::st(A.accumulate ? Store<TF>::ld(fr[u]) + A.scale * Fv[q][k] : A.scale * Fv[q][k]);
        }
    }
}

constexpr int kFwdK = 8;

}  // namespace

template <class TF, class TG>
int project_tma_t(const petl_geom& G, const TF* f, TG* g, const ViewRange& vr, const TG* meas, const Tables& T,
                  cudaStream_t st)
{
    constexpr int FBOXW = fboxw<TF>();
    constexpr int EB = int(sizeof(TF));
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return 0;
    // volume rows a multiple of 16 bytes (TMA strides), 16-byte aligned base
    if ((G.numX * EB) % 16 != 0 || (reinterpret_cast<uintptr_t>(f) & 15) != 0 || G.numY > 4096)
        return kNotApplicable;
    const double step = double(G.T_v1) * plane_ymax(G) / double(G.T_z);  // shift change per slope
    if (shift_spread(FV - 1, step) > FDMAX) return kNotApplicable;
    const int nrb = FROWS + shift_spread(FSL - 1, step) + 1;
    if (nrb > 256) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;
    CUtensorMap map;
    const uint64_t dims[3] = {uint64_t(G.numX), uint64_t(G.numY), uint64_t(G.numZ)};
    const uint64_t strides[2] = {uint64_t(G.numX) * EB, uint64_t(G.numX) * G.numY * EB};
    const uint32_t box[3] = {uint32_t(FBOXW), 1u, uint32_t(nrb)};
    if (!encode_tensor_map(&map, f, 3, dims, strides, box, EB)) return kNotApplicable;

    FwdTmaArgs A{};
    A.G = G;
    A.vr = vr;
    A.n_colblk = int(ceil_div(G.N_u0, FCOLS));
    A.nrb = nrb;
    A.fstride = (nrb * FBOXW * EB + 127) & ~127;
    A.xstride = (nrb + FDMAX) * FCOLS;
    A.T = T;
    A.err = err;
    A.wait_limit = wait_limit();
    // up to 4 planes in flight; prefer a footprint that leaves room for two
    // CTAs per SM, else the largest ring that fits one
    auto bytes = [&](int nf) {
        return size_t(nf) * A.fstride + size_t(4) * A.xstride * 4 + size_t(1 + FSL) * G.numY * sizeof(Shift) +
               size_t(nf) * 8 + 2 * 4 + size_t(G.numY) * 2;
    };
    A.nf = 0;
    for (int nf = 4; nf >= 2 && !A.nf; nf--)
        if (bytes(nf) <= 113 * 1024) A.nf = nf;
    for (int nf = 4; nf >= 2 && !A.nf; nf--)
        if (bytes(nf) <= 227 * 1024) A.nf = nf;
    if (!A.nf) return kNotApplicable;
    const size_t smem = bytes(A.nf);
    auto kern = k_fwd_tma<kFwdK, TF, TG>;
    PETL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 grid(unsigned(n_v0), ceil_div(nv1, FSL), unsigned(A.n_colblk) * ceil_div(G.N_u1, FROWS));
    kern<<<grid, 32 * FGV * (FROWS / kFwdK), smem, st>>>(map, g, meas, A);
    PETL_LAUNCH_CHECK("project_tma");
    return 0;
}

template <class TG, class TF>
int backproject_tma_t(const petl_geom& G, const TG* g, TF* f, int mode, int accumulate, float scale,
                      const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    constexpr int EB = int(sizeof(TG));
    const int NU0 = G.N_u0;
    if ((reinterpret_cast<uintptr_t>(g) & 15) != 0) return kNotApplicable;
    // tensor-map staging when the rows are multiples of 16 bytes and fit one
    // 256-element box; FP32 planograms with even rows otherwise take bulk
    // copies of row pairs (up to 512 columns)
    const bool tensor = (NU0 * EB) % 16 == 0 && NU0 <= 256 && G.numX <= 256;
    const bool bulk = !tensor && EB == 4 && NU0 % 2 == 0 && G.N_u1 % 2 == 0 && NU0 <= 512 && G.numX <= 512;
    if (!tensor && !bulk) return kNotApplicable;
    const int pg = std::max(NU0, G.numX) <= 256 ? 2 : 1;
    const int np = BPT * pg;
    if (vr.iv1_end - vr.iv1_begin > BV1CAP) return kNotApplicable;
    const double step = double(std::max(std::fabs(G.v1_0), std::fabs(G.v1_0 + (G.N_v1 - 1) * G.T_v1))) *
                        double(G.T_x) / double(G.T_z);  // shift change per plane
    if (shift_spread(BPT - 1, step) > BDW) return kNotApplicable;
    const int brb = BWN + shift_spread(np - 1, step);
    if (brb > 254) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (tensor) {
        const uint64_t dims[4] = {uint64_t(NU0), uint64_t(G.N_u1), uint64_t(G.N_v0), uint64_t(G.N_v1)};
        const uint64_t strides[3] = {uint64_t(NU0) * EB, uint64_t(NU0) * G.N_u1 * EB,
                                     uint64_t(NU0) * G.N_u1 * G.N_v0 * EB};
        const uint32_t box[4] = {uint32_t(NU0), uint32_t(brb), 1u, 1u};
        if (!encode_tensor_map(&map, g, 4, dims, strides, box, EB)) return kNotApplicable;
    }

    BwdTmaArgs A{};
    A.G = G;
    A.vr = vr;
    A.ncw = int(ceil_div(std::max(NU0, G.numX), 32));
    A.brb = brb;
    // bulk copies stage whole row pairs: up to two rows more than the window
    A.sstride = ((brb + (bulk ? 2 : 0)) * NU0 * EB + 127) & ~127;
    A.accumulate = accumulate;
    A.scale = scale;
    A.T = T;
    A.err = err;
    A.wait_limit = wait_limit();
    // as many ring stages as fit (copies from DRAM need several in flight)
    A.max_views = vr.n_v0(G.N_v0);
    const size_t fixed = size_t(np) * BK * NU0 * 4 + size_t(BV1CAP) * np * 8 + size_t(BV1CAP) * np * 4 +
                         size_t(A.max_views) * np * sizeof(Shift) + size_t(BV1CAP) * 4 * 4 +
                         size_t(BV1CAP) * pg * 4 * 2 + size_t(BV1CAP) * 4 + 2 * BNSMAX * 8 + 8 + BNSMAX * 4 + 16;
    A.ns = int(std::min<size_t>(BNSMAX, (227 * 1024 - std::min<size_t>(fixed, 227 * 1024)) / size_t(A.sstride)));
    if (A.ns < 2) return kNotApplicable;
    const size_t smem = size_t(A.ns) * A.sstride + fixed;
    const int threads = 32 * A.ncw * pg;
    dim3 grid(ceil_div(G.numY, np), ceil_div(G.numZ, BK));
    const bool adj = mode == PETL_BP_ADJOINT;
    auto kern = adj ? k_bwd_tma<true, 0, TG, TF, false, 2> : k_bwd_tma<false, 0, TG, TF, false, 2>;
    if (tensor && NU0 == 256) kern = adj ? k_bwd_tma<true, 256, TG, TF, false, 2> : k_bwd_tma<false, 256, TG, TF, false, 2>;
    if constexpr (sizeof(TG) == 4) {
        if (bulk)
            kern = pg == 2 ? (adj ? k_bwd_tma<true, 0, TG, TF, true, 2> : k_bwd_tma<false, 0, TG, TF, true, 2>)
                           : (adj ? k_bwd_tma<true, 0, TG, TF, true, 1> : k_bwd_tma<false, 0, TG, TF, true, 1>);
    }
    PETL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    kern<<<grid, threads, smem, st>>>(map, g, f, A);
    PETL_LAUNCH_CHECK("backproject_tma");
    return 0;
}

int project_tma(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                const Tables& T, cudaStream_t st)
{
    // the split form (x-shift pass + z-tap kernel) first; dispatch 3 keeps
    // the fused kernel
    if (dispatch_mode() != 3) {
        const int rc = project_split(G, f, g, vr, meas, T, st);
        if (rc != kNotApplicable) return rc;
    }
    return project_tma_t<float, float>(G, f, g, vr, meas, T, st);
}

int backproject_tma(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                    const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    // the split form (z-gather into scratch + x-gather) first; dispatch 3
    // keeps the single-pass kernel
    if (dispatch_mode() != 3) {
        const int rc = backproject_split(G, g, f, mode, accumulate, scale, vr, T, st);
        if (rc != kNotApplicable) return rc;
    }
    return backproject_tma_t<float, float>(G, g, f, mode, accumulate, scale, vr, T, st);
}

int project_tma_bf16(const petl_geom& G, const __nv_bfloat16* f, __nv_bfloat16* g, const ViewRange& vr,
                     const __nv_bfloat16* meas, const Tables& T, cudaStream_t st)
{
    if (dispatch_mode() != 3) {
        const int rc = project_split_bf16(G, f, g, vr, meas, T, st);
        if (rc != kNotApplicable) return rc;
    }
    return project_tma_t<__nv_bfloat16, __nv_bfloat16>(G, f, g, vr, meas, T, st);
}

int backproject_tma_bf16(const petl_geom& G, const __nv_bfloat16* g, float* f, int mode, int accumulate, float scale,
                         const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    if (dispatch_mode() != 3) {
        const int rc = backproject_split_bf16(G, g, f, mode, accumulate, scale, vr, T, st);
        if (rc != kNotApplicable) return rc;
    }
    return backproject_tma_t<__nv_bfloat16, float>(G, g, f, mode, accumulate, scale, vr, T, st);
}

}  // namespace shear
}  // namespace petl
