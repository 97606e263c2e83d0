// TMA-staged shear-warp projector and backprojectors (psi = 0, voxel pitch
// equal to the bin pitch).  They compute the operator of the first-generation
// kernels in projector_shear.cu (the shear-warp form of the reference
// footprint, src/projectors.cu:131-185 forward and :240-377 backward); only
// the staging and the register blocking differ.
//
// Forward, k_fwd_tma: one CTA per (view v0, 16 slopes v1, 32 rows u1, 64
// columns u0).  For each plane y that reaches the tile, one thread starts a
// TMA copy of the raw volume rows the tile needs (68 columns x nrb rows of
// plane y; whatever lies outside the volume arrives as zeros) two planes
// ahead of use.  The CTA interpolates the rows in x into shared memory once,
// then each warp applies the z interpolation of its 4 slopes from a single
// register window of K + 4 rows (the integer shifts of 4 consecutive slopes
// differ by at most 3 rows), two columns per lane with packed FP32 FMAs.
//
// Backward, k_bwd_tma<ADJ>: one CTA per (8 planes y, 8 rows z, all columns).
// For every (view v0, slope v1) whose rows reach the tile, one thread starts a
// TMA copy of the planogram rows the tile needs (N_u0 columns x brb rows) into
// a 4-stage ring.  Each thread sums, for its 4 planes and 2 columns, the
// z-interpolated rows of every slope from one register window (the shifts of
// 4 consecutive planes differ by at most 2 rows); after each view the x shift
// goes through shared memory into voxel accumulators held in registers.  Each
// voxel is owned by one CTA: no atomics, one write at the end.
//
// Every wait on a copy is bounded; a wait that gives up sets the device error
// word, and the CTA drains its copies in flight and stops without writing.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"
#include "tma.cuh"

namespace petl {
namespace shear {

namespace {

enum : int { kErrLayout = 2 };  // a host-side bound on the shift spread did not hold

__device__ __forceinline__ float2 dup(float a) { return make_float2(a, a); }

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ===========================================================================
// forward
// ===========================================================================
constexpr int FV = 4;              // slopes per warp
constexpr int FGV = 4;             // warps along v1
constexpr int FSL = FV * FGV;      // slopes per CTA
constexpr int FROWS = 32;          // rows per CTA
constexpr int FCOLS = 64;          // columns per CTA, two per lane
constexpr int FBOXW = FCOLS + 4;   // staged raw columns: 64 + 1 tap + 3 for 16-byte alignment
constexpr int FDMAX = 3;           // largest shift difference among a warp's slopes

struct FwdTmaArgs {
    petl_geom G;
    ViewRange vr;
    int n_colblk;  // ceil(N_u0 / 64)
    int nrb;       // staged rows per plane (32 + CTA shift spread + 1, bounded on the host)
    int fstride;   // floats per raw buffer
    int xstride;   // floats per interpolated buffer
    Tables T;
    int* err;
};

struct FwdPlane {
    int cx;     // volume column of tile column 0 (before the x tap)
    int wlo;    // volume row of staged row 0
    int nr;     // staged rows used
    int dzmin;  // smallest z shift among the CTA's slopes
    float wx;   // x tap weight
};

// Plane geometry of a forward tile: the z shift is monotone in v1, so the
// extreme shifts sit at the first and last slope.
__device__ __forceinline__ FwdPlane fwd_plane(const FwdTmaArgs& A, int iv0, int v1a, int v1b, int col0, int row0,
                                              int y)
{
    const int NY = A.G.numY;
    const Shift xs = A.T.xt[size_t(iv0) * NY + y];
    const int da = A.T.zt[size_t(v1a) * NY + y].d, db = A.T.zt[size_t(v1b) * NY + y].d;
    FwdPlane p;
    p.dzmin = min(da, db);
    p.cx = col0 + xs.d;
    p.wx = xs.w;
    p.wlo = row0 + p.dzmin;
    p.nr = FROWS + (max(da, db) - p.dzmin) + 1;
    return p;
}

template <int O, int K>
__device__ __forceinline__ void fwd_taps(float2 (&acc)[K], const float2 (&W)[K + FDMAX + 1], float2 w0, float2 w1)
{
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = __ffma2_rn(w1, W[k + O + 1], __ffma2_rn(w0, W[k + O], acc[k]));
}

template <int K>
__global__ void __launch_bounds__(32 * FGV * (FROWS / K), 1)
k_fwd_tma(const __grid_constant__ CUtensorMap fmap, float* __restrict__ g, const float* __restrict__ meas,
          const FwdTmaArgs A)
{
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
    const int rowblk = blockIdx.z / A.n_colblk, colblk = blockIdx.z % A.n_colblk;
    const int cta_row0 = rowblk * FROWS, col0 = colblk * FCOLS;
    const int v1w = v1a + gv * FV;       // first slope of this warp
    const int row0 = cta_row0 + gr * K;  // first row of this warp
    const int NY = G.numY, NZ = G.numZ, NX = G.numX;

    float* Fr = reinterpret_cast<float*>(smem);  // [2][nrb][68] raw rows (TMA)
    float* Xs = Fr + 2 * A.fstride;              // [2][nrb + 3][64] x-interpolated rows
    uint64_t* bar = reinterpret_cast<uint64_t*>(Xs + 2 * A.xstride);
    int* s_n = reinterpret_cast<int*>(bar + 2);
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
        const int v1 = v1w + j;
        if (v1 <= v1b) {
            const int2 u = A.T.ub1[v1];
            if (!(row0 > u.y || row0 + K - 1 < u.x)) wmask |= 1u << j;
        }
    }

    float2 acc[FV][K];
#pragma unroll
    for (int j = 0; j < FV; j++)
#pragma unroll
        for (int k = 0; k < K; k++) acc[j][k] = make_float2(0.0f, 0.0f);

    if (live) {  // CTA-uniform
        // planes whose staged window meets the volume, compacted in order
        if (warp == 0) {
            int n = 0;
            for (int yb = 0; yb < NY; yb += 32) {
                const int y = yb + lane;
                bool ok = false;
                if (y < NY) {
                    const FwdPlane p = fwd_plane(A, iv0, v1a, v1b, col0, cta_row0, y);
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
                mbar_init(&bar[0], 1);
                mbar_init(&bar[1], 1);
                fence_barrier_init();
            }
        }
        __syncthreads();
        const int nlive = s_n[0];
        const uint32_t box_bytes = uint32_t(FBOXW) * uint32_t(A.nrb) * 4u;
        int issued = 0;  // thread 0 only
        auto issue = [&](int li) {
            const int y = plist[li];
            const FwdPlane p = fwd_plane(A, iv0, v1a, v1b, col0, cta_row0, y);
            const int b = li & 1;
            mbar_arrive_expect_tx(&bar[b], box_bytes);
            // x rounded down to a multiple of 4 floats: TMA needs 16-byte aligned starts
            tma_load_3d(Fr + b * A.fstride, &fmap, &bar[b], p.cx & ~3, y, p.wlo);
        };
        if (tid == 0) {
            for (; issued < 2 && issued < nlive; issued++) issue(issued);
        }

        bool dead = false;
        int li = 0;
        for (; li < nlive; li++) {
            const int b = li & 1;
            const int y = plist[li];
            const FwdPlane p = fwd_plane(A, iv0, v1a, v1b, col0, cta_row0, y);
            if (!dead) dead = !mbar_wait(&bar[b], uint32_t((li >> 1) & 1), A.err);
            // stage A: x interpolation of the staged rows (one column per lane)
            {
                const float* F = Fr + b * A.fstride + (p.cx - (p.cx & ~3));
                float* X = Xs + b * A.xstride;
                const float w1 = p.wx, w0 = 1.0f - p.wx;
                for (int e = tid; e < p.nr * FCOLS; e += NT) {
                    const float* fr = F + (e >> 6) * FBOXW + (e & 63);
                    X[e] = fmaf(w1, fr[1], w0 * fr[0]);
                }
            }
            if (__syncthreads_or(dead)) break;
            // every thread is done with raw buffer b: stage plane li + 2 into it
            if (tid == 0 && issued < nlive) {
                fence_proxy_async_smem();
                issue(issued);
                issued++;
            }
            // stage B: z interpolation of this warp's slopes from one window
            if (wmask) {  // warp-uniform
                Shift zs[FV];
                int base = 1 << 30;
#pragma unroll
                for (int j = 0; j < FV; j++) {
                    zs[j] = Shift{0, 0.0f};
                    if ((wmask >> j) & 1u) {
                        zs[j] = A.T.zt[size_t(v1w + j) * NY + y];
                        base = min(base, zs[j].d);
                    }
                }
                const int xr0 = row0 - cta_row0 + base - p.dzmin;  // staged row of window row 0
                const int iz0 = p.wlo + xr0;                        // its volume row
                if (base < p.dzmin) {  // the shifts are monotone in v1; never read before the buffer
                    atomicOr(A.err, kErrLayout);
                } else if (iz0 + WN - 1 >= 0 && iz0 < NZ) {
                    const float* Xr = Xs + b * A.xstride + xr0 * FCOLS + 2 * lane;
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
                }
            }
        }
        if (li < nlive) {
            // a wait gave up: drain the copies still in flight, write nothing
            if (tid == 0)
                for (int q = li; q < issued; q++) mbar_wait(&bar[q & 1], uint32_t((q >> 1) & 1), nullptr);
            return;
        }
    }

    // epilogue: scale, ray masks, optional MLEM ratio
    const int colA = col0 + 2 * lane;
    const bool pairs = (G.N_u0 & 1) == 0;  // float2 accesses stay 8-byte aligned
#pragma unroll
    for (int j = 0; j < FV; j++) {
        const int v1 = v1w + j;
        if (v1 > v1b) continue;
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
                    const float2 m = __ldg(reinterpret_cast<const float2*>(meas + o));
                    val = make_float2(ratio_rule(m.x, val.x), ratio_rule(m.y, val.y));
                }
                *reinterpret_cast<float2*>(g + o) = val;
            } else {
                if (colA < G.N_u0) g[o] = meas ? ratio_rule(__ldg(meas + o), val.x) : val.x;
                if (colA + 1 < G.N_u0) g[o + 1] = meas ? ratio_rule(__ldg(meas + o + 1), val.y) : val.y;
            }
        }
    }
}

// ===========================================================================
// backward
// ===========================================================================
constexpr int BK = 8;               // z rows per CTA
constexpr int BPT = 4;              // planes per thread
constexpr int BPG = 2;              // plane groups
constexpr int BNP = BPT * BPG;      // planes per CTA
constexpr int BDW = 2;              // largest shift difference among a thread's planes
constexpr int BWN = BK + BDW + 1;   // register window rows
constexpr int BNS = 4;              // copy ring stages
constexpr int BV1CAP = 96;          // slopes held in the per-CTA tables

struct BwdTmaArgs {
    petl_geom G;
    ViewRange vr;
    int ncw;      // column warps per plane group (64 columns each)
    int brb;      // staged rows per view (>= BWN + CTA shift spread, bounded on the host)
    int sstride;  // floats per ring stage
    int accumulate;
    float scale;
    Tables T;
    int* err;
};

// z taps of one plane: Z[k] += w1 g[row k of tap 1] + w0 g[row k of tap 0],
// window row O + k holding tap 1 and O + k + 1 tap 0.  MASK applies per-row
// 0/1 factors: vm (window rows that hold visible bins, the adjoint's bin mask)
// and om (output rows inside the reference backprojector's voxel test).
template <int O, bool MASK>
__device__ __forceinline__ void bwd_taps(float2 (&Z)[BK], const float2 (&W)[BWN], float2 w0, float2 w1, uint32_t vm,
                                         uint32_t om)
{
#pragma unroll
    for (int k = 0; k < BK; k++) {
        if (MASK) {
            const float a = ((vm >> (O + k)) & (om >> k) & 1u) ? 1.0f : 0.0f;
            const float b = ((vm >> (O + k + 1)) & (om >> k) & 1u) ? 1.0f : 0.0f;
            Z[k] = __ffma2_rn(make_float2(w1.x * a, w1.y * a), W[O + k],
                              __ffma2_rn(make_float2(w0.x * b, w0.y * b), W[O + k + 1], Z[k]));
        } else {
            Z[k] = __ffma2_rn(w1, W[O + k], __ffma2_rn(w0, W[O + k + 1], Z[k]));
        }
    }
}

template <bool ADJ>
__global__ void __launch_bounds__(256, 1)
k_bwd_tma(const __grid_constant__ CUtensorMap gmap, float* __restrict__ f, const BwdTmaArgs A)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    const int cw = warp % A.ncw, pg = warp / A.ncw;
    const int p0 = blockIdx.x * BNP;  // first plane of the CTA
    const int r0 = blockIdx.y * BK;   // first z row of the CTA
    const int u = cw * 64 + 2 * lane; // first of this thread's two columns
    const int NY = G.numY, NX = G.numX, NZ = G.numZ, NU0 = G.N_u0, NU1 = G.N_u1;
    const int n_v0 = A.vr.n_v0(G.N_v0);

    float* ring = reinterpret_cast<float*>(smem);                         // [BNS][brb][NU0]
    float* Zs = ring + BNS * A.sstride;                                   // [BNP][BK][NU0]
    float4* Wt = reinterpret_cast<float4*>(Zs + BNP * BK * NU0);          // [BV1CAP][BNP]
    float* s_w = reinterpret_cast<float*>(Wt + BV1CAP * BNP);             // [BV1CAP][BNP]
    int* s_v1 = reinterpret_cast<int*>(s_w + BV1CAP * BNP);               // [BV1CAP]
    int* s_grow = s_v1 + BV1CAP;                                          // [BV1CAP]
    uint32_t* s_code = reinterpret_cast<uint32_t*>(s_grow + BV1CAP);      // [BV1CAP]
    uint32_t* s_wb = s_code + BV1CAP;                                     // [BV1CAP]
    uint64_t* full = reinterpret_cast<uint64_t*>(s_wb + BV1CAP);          // [BNS]
    uint64_t* empty = full + BNS;                                         // [BNS]
    int* s_n = reinterpret_cast<int*>(empty + BNS);

    // ---- per-CTA slope tables (warp 0): for every slope whose rows reach the
    // tile, the staged g row, per plane the window offset and mode (0 none,
    // 1 full, 2 masked rows), per plane group the window base row.
    if (warp == 0) {
        int n = 0;
        for (int vb = A.vr.iv1_begin; vb < A.vr.iv1_end; vb += 32) {
            const int v1 = vb + lane;
            bool ok = false;
            uint32_t code = 0, wbs = 0;
            int grow = 0;
            float wz[BNP];
            if (v1 < A.vr.iv1_end) {
                int dz[BNP];
                int dmin = 1 << 30, dmax = -(1 << 30);
#pragma unroll
                for (int p = 0; p < BNP; p++) {
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
                int mode[BNP];
#pragma unroll
                for (int p = 0; p < BNP; p++) {
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
                }
                bool bad = dmax - dmin > A.brb - BWN;
#pragma unroll
                for (int q = 0; q < BPG; q++) {
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
                    s_wb[idx] = wbs;
#pragma unroll
                    for (int p = 0; p < BNP; p++) s_w[idx * BNP + p] = wz[p];
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
            for (int s = 0; s < BNS; s++) {
                mbar_init(&full[s], 1);
                mbar_init(&empty[s], nwarps);
            }
            fence_barrier_init();
        }
    }
    __syncthreads();
    const int nlive = s_n[0];
    const long long total = (long long)n_v0 * nlive;

    // weights of view v0: (S w0, S w0, S w1, S w1) per live slope and plane
    auto weights = [&](int v0) {
        for (int e = tid; e < nlive * BNP; e += blockDim.x) {
            const int li = e / BNP;
            const float S = A.T.S[size_t(s_v1[li]) * G.N_v0 + v0];
            const float w = s_w[e];
            const float w1 = S * w, w0 = S * (1.0f - w);
            Wt[e] = make_float4(w0, w0, w1, w1);
        }
    };
    const uint32_t box_bytes = uint32_t(NU0) * uint32_t(A.brb) * 4u;
    long long issued = 0;  // thread 0 only
    bool dead = false;
    // start the copy of stage j once every warp has released its ring slot
    auto issue = [&](long long j) {
        const int s = int(j % BNS);
        const int li = int(j % nlive);
        const int v0 = A.vr.iv0_first + int(j / nlive) * A.vr.iv0_step;
        if (j >= BNS && !mbar_wait(&empty[s], uint32_t(((j / BNS) - 1) & 1), A.err)) return false;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full[s], box_bytes);
        tma_load_4d(ring + s * A.sstride, &gmap, &full[s], 0, s_grow[li], v0, s_v1[li]);
        return true;
    };
    if (tid == 0)
        for (; issued < BNS - 1 && issued < total; issued++) issue(issued);
    if (n_v0 > 0) weights(A.vr.iv0_first);
    __syncthreads();

    float2 Fv[BPT][BK];  // voxel accumulators (unscaled)
    float2 Z[BPT][BK];   // z-interpolated sums of the current view
#pragma unroll
    for (int q = 0; q < BPT; q++)
#pragma unroll
        for (int k = 0; k < BK; k++) {
            Fv[q][k] = make_float2(0.0f, 0.0f);
            Z[q][k] = make_float2(0.0f, 0.0f);
        }

    bool aborted = false;
    const bool ucol = u < NU0;
    long long it = 0;
    for (int iv = 0; iv < n_v0 && !aborted; iv++) {
        const int v0 = A.vr.iv0_first + iv * A.vr.iv0_step;
        for (int li = 0; li < nlive; li++, it++) {
            if (tid == 0 && issued < total && !dead) {
                if (issue(issued))
                    issued++;
                else
                    dead = true;
            }
            const int s = int(it % BNS);
            if (!dead) dead = !mbar_wait(&full[s], uint32_t((it / BNS) & 1), A.err);
            const uint32_t code = s_code[li] >> (16 * pg);  // this group's 4 planes
            if (ucol && (code & 0x3333u)) {
                const int wb = (s_wb[li] >> (8 * pg)) & 0xff;
                const float* Gs = ring + s * A.sstride + wb * NU0 + u;
                float2 W[BWN];
#pragma unroll
                for (int i = 0; i < BWN; i++) W[i] = *reinterpret_cast<const float2*>(Gs + i * NU0);
                const float4* Wl = Wt + li * BNP + pg * BPT;
#pragma unroll
                for (int q = 0; q < BPT; q++) {
                    const uint32_t c = (code >> (4 * q)) & 15u;
                    if (!(c & 3u)) continue;
                    const float4 w = Wl[q];
                    const float2 w0 = make_float2(w.x, w.y), w1 = make_float2(w.z, w.w);
                    const int o = int(c >> 2);
                    if ((c & 3u) == 1u) {
                        switch (o) {
                            case 0: bwd_taps<0, false>(Z[q], W, w0, w1, 0u, 0u); break;
                            case 1: bwd_taps<1, false>(Z[q], W, w0, w1, 0u, 0u); break;
                            default: bwd_taps<2, false>(Z[q], W, w0, w1, 0u, 0u); break;
                        }
                    } else {
                        // rows at the edge of the visible range: per-row masks
                        uint32_t vm = 0xffffffffu, om = 0xffffffffu;
                        const int v1 = s_v1[li];
                        if (ADJ) {
                            const int2 ub1 = A.T.ub1[v1];
                            const int gr0 = s_grow[li] + wb;  // g row of window row 0
                            vm = 0;
#pragma unroll
                            for (int i = 0; i < BWN; i++)
                                if (gr0 + i >= ub1.x && gr0 + i <= ub1.y) vm |= 1u << i;
                        } else {
                            const int2 zv = A.T.zvis[size_t(v1) * NY + p0 + pg * BPT + q];
                            om = 0;
#pragma unroll
                            for (int k = 0; k < BK; k++)
                                if (r0 + k >= zv.x && r0 + k <= zv.y) om |= 1u << k;
                        }
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
                        float2 z = Z[q][k];
                        if (ADJ) {
                            if (u < u0r.x || u > u0r.y) z.x = 0.0f;
                            if (u + 1 < u0r.x || u + 1 > u0r.y) z.y = 0.0f;
                        }
                        *reinterpret_cast<float2*>(Zs + ((pg * BPT + q) * BK + k) * NU0 + u) = z;
                    }
                    Z[q][k] = make_float2(0.0f, 0.0f);
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
            const Shift xs = A.T.xt[size_t(v0) * NY + y];
            const float wx1 = xs.w, wx0 = 1.0f - xs.w;
            const int j0 = u - xs.d;  // Z column of tap 0 for voxel column u
#pragma unroll
            for (int k = 0; k < BK; k++) {
                const float* zr = Zs + ((pg * BPT + q) * BK + k) * NU0;
                const float zm = (j0 - 1 >= 0 && j0 - 1 < NU0) ? zr[j0 - 1] : 0.0f;
                const float z0 = (j0 >= 0 && j0 < NU0) ? zr[j0] : 0.0f;
                const float zp = (j0 + 1 >= 0 && j0 + 1 < NU0) ? zr[j0 + 1] : 0.0f;
                Fv[q][k].x += fmaf(wx1, zm, wx0 * z0);
                Fv[q][k].y += fmaf(wx1, z0, wx0 * zp);
            }
        }
        if (iv + 1 < n_v0) weights(v0 + A.vr.iv0_step);
        __syncthreads();
    }
    if (aborted) {
        // a wait gave up: drain the copies still in flight, write nothing
        if (tid == 0)
            for (long long j = std::max(0LL, issued - BNS); j < issued; j++)
                mbar_wait(&full[j % BNS], uint32_t((j / BNS) & 1), nullptr);
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
            float* fr = f + (size_t(z) * NY + y) * NX;
            if (u < NX) fr[u] = A.accumulate ? fr[u] + A.scale * Fv[q][k].x : A.scale * Fv[q][k].x;
            if (u + 1 < NX) fr[u + 1] = A.accumulate ? fr[u + 1] + A.scale * Fv[q][k].y : A.scale * Fv[q][k].y;
        }
    }
}

double plane_ymax(const petl_geom& G)
{
    return std::max(std::fabs(double(G.y_0)), std::fabs(double(G.y_0) + (G.numY - 1) * double(G.T_x)));
}

// Upper bound on the difference of the integer z shifts of slopes (or planes)
// n steps apart: the exact shifts differ by at most n * step, their floors by
// at most floor(n * step) + 1 (with a relative margin for the float inputs).
int shift_spread(int n, double step) { return int(std::floor(double(n) * step * (1.0 + 1e-6))) + 1; }

constexpr int kFwdK = 16;

}  // namespace

int project_tma(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                const Tables& T, cudaStream_t st)
{
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return 0;
    if (G.numX % 4 != 0 || (reinterpret_cast<uintptr_t>(f) & 15) != 0 || G.numY > 4096) return kNotApplicable;
    const double step = double(G.T_v1) * plane_ymax(G) / double(G.T_z);  // shift change per slope
    if (shift_spread(FV - 1, step) > FDMAX) return kNotApplicable;
    const int nrb = FROWS + shift_spread(FSL - 1, step) + 1;
    if (nrb > 256) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;
    CUtensorMap map;
    const uint64_t dims[3] = {uint64_t(G.numX), uint64_t(G.numY), uint64_t(G.numZ)};
    const uint64_t strides[2] = {uint64_t(G.numX) * 4, uint64_t(G.numX) * G.numY * 4};
    const uint32_t box[3] = {uint32_t(FBOXW), 1u, uint32_t(nrb)};
    if (!encode_tensor_map(&map, f, 3, dims, strides, box)) return kNotApplicable;

    FwdTmaArgs A{};
    A.G = G;
    A.vr = vr;
    A.n_colblk = int(ceil_div(G.N_u0, FCOLS));
    A.nrb = nrb;
    A.fstride = ((nrb * FBOXW * 4 + 127) & ~127) / 4;
    A.xstride = (nrb + FDMAX) * FCOLS;
    A.T = T;
    A.err = err;
    const size_t smem = size_t(2) * A.fstride * 4 + size_t(2) * A.xstride * 4 + 2 * 8 + 2 * 4 + size_t(G.numY) * 2;
    if (smem > 227 * 1024) return kNotApplicable;
    auto kern = k_fwd_tma<kFwdK>;
    PETL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 grid(unsigned(n_v0), ceil_div(nv1, FSL), unsigned(A.n_colblk) * ceil_div(G.N_u1, FROWS));
    kern<<<grid, 32 * FGV * (FROWS / kFwdK), smem, st>>>(map, g, meas, A);
    PETL_LAUNCH_CHECK("project_tma");
    return 0;
}

int backproject_tma(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                    const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    const int NU0 = G.N_u0;
    if (NU0 % 4 != 0 || NU0 > 256 || G.numX > 256 || (reinterpret_cast<uintptr_t>(g) & 15) != 0)
        return kNotApplicable;
    if (vr.iv1_end - vr.iv1_begin > BV1CAP) return kNotApplicable;
    const double step = double(std::max(std::fabs(G.v1_0), std::fabs(G.v1_0 + (G.N_v1 - 1) * G.T_v1))) *
                        double(G.T_x) / double(G.T_z);  // shift change per plane
    if (shift_spread(BPT - 1, step) > BDW) return kNotApplicable;
    const int brb = BWN + shift_spread(BNP - 1, step);
    if (brb > 256) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;
    CUtensorMap map;
    const uint64_t dims[4] = {uint64_t(NU0), uint64_t(G.N_u1), uint64_t(G.N_v0), uint64_t(G.N_v1)};
    const uint64_t strides[3] = {uint64_t(NU0) * 4, uint64_t(NU0) * G.N_u1 * 4,
                                 uint64_t(NU0) * G.N_u1 * G.N_v0 * 4};
    const uint32_t box[4] = {uint32_t(NU0), uint32_t(brb), 1u, 1u};
    if (!encode_tensor_map(&map, g, 4, dims, strides, box)) return kNotApplicable;

    BwdTmaArgs A{};
    A.G = G;
    A.vr = vr;
    A.ncw = int(ceil_div(std::max(NU0, G.numX), 64));
    A.brb = brb;
    A.sstride = ((brb * NU0 * 4 + 127) & ~127) / 4;
    A.accumulate = accumulate;
    A.scale = scale;
    A.T = T;
    A.err = err;
    const size_t smem = size_t(BNS) * A.sstride * 4 + size_t(BNP) * BK * NU0 * 4 + size_t(BV1CAP) * BNP * 16 +
                        size_t(BV1CAP) * BNP * 4 + size_t(BV1CAP) * 4 * 4 + 2 * BNS * 8 + 16;
    if (smem > 227 * 1024) return kNotApplicable;
    const int threads = 32 * A.ncw * BPG;
    dim3 grid(ceil_div(G.numY, BNP), ceil_div(G.numZ, BK));
    if (mode == PETL_BP_ADJOINT) {
        PETL_CUDA(cudaFuncSetAttribute(k_bwd_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        k_bwd_tma<true><<<grid, threads, smem, st>>>(map, f, A);
    } else {
        PETL_CUDA(cudaFuncSetAttribute(k_bwd_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        k_bwd_tma<false><<<grid, threads, smem, st>>>(map, f, A);
    }
    PETL_LAUNCH_CHECK("backproject_tma");
    return 0;
}

}  // namespace shear
}  // namespace petl
