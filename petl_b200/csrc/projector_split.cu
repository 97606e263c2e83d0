// Split forward projector (psi = 0, voxel pitch equal to the bin pitch).
//
// The shear-warp form of the reference footprint (src/projectors.cu:131-185,
// see projector_shear.cu) adds, for every plane y,
//   g[v1][v0][iu1][iu0] += wz0 X[iu1 + dz][iu0] + wz1 X[iu1 + dz + 1][iu0]
// where X is plane y of the volume interpolated in x by the shift of view v0:
//   X_v0[y][z][c] = (1 - wx) f[z][y][c + dx] + wx f[z][y][c + dx + 1].
// project_tma computes X inside every CTA (stage A) between two CTA barriers
// per plane pair.  Here the two stages are separate kernels:
//
// * k_xshift writes X for a chunk of views into FP32 scratch, [view][y][z][c]
//   (memory bound: one write of a volume per view; each volume row is read
//   once per chunk);
// * k_fwd_zsum applies the z taps.  CTA = one view x 16 slopes x 32 rows x 64
//   columns, 16 warps of 4 slopes x 8 rows x 2 columns per lane.  The staged
//   rows of each plane arrive by a tiled TMA copy (no multicast) into a ring
//   of two stages of two planes with full/empty mbarriers; the copy of a stage is
//   started by a rotating warp once every warp has released the slot, so no
//   CTA-wide barrier sits in the plane loop.  The window offset, tap offsets
//   and weights of every (plane, slope group) are tabulated once per CTA.
//   The tap offsets of a warp's four consecutive slopes move by at most one
//   row from slope to slope, so they form one of 15 monotone patterns: one
//   dispatch per plane selects a fully unrolled form (four per-slope
//   dispatches measured 10 % slower); other groups take the per-slope form.
//
// Both kernels do the float operations of project_tma in the same order (x
// taps fmaf(w1, b, w0 * a); per ray, the z taps of the live planes in
// ascending y, tap 0 then tap 1), so the two paths agree bit for bit.
//
// A launch serves the views of one call or, for the server's batched steps,
// of up to kMaxMembers requests of one geometry (Members: per-member
// volumes, planograms and view subsets; member b's views in scratch slots
// b * nvm + v).  The kernels are compiled for one member (plain calls) and
// for up to kMaxMembers.
//
// Every wait is bounded: a wait that gives up sets the device error word,
// the CTA drains its copies in flight and returns without writing.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {
namespace shear {

namespace {

constexpr int ZV = 4;                 // slopes per warp
constexpr int ZK = 8;                 // rows per warp
constexpr int ZSG = 4;                // slope groups of a full block (warps along v1)
constexpr int ZSL = ZV * ZSG;         // slopes of a full block
constexpr int ZCOLS = 64;             // columns per CTA, two per lane
constexpr int ZWARPS = 16;
constexpr int ZNT = 32 * ZWARPS;
constexpr int ZDMAX = 3;              // largest shift difference among a warp's slopes
constexpr int ZWN = ZK + ZDMAX + 1;   // register window rows
// ring stages (of two planes each): three measured 0.9 % faster than two at
// the 256x256x128 workload once the tap offsets were dispatched per plane
// (before that, deeper rings ran 1-3 % slower)
constexpr int ZNSMAX = 3;
constexpr int ZMAXPLANES = 1024;      // planes the per-CTA tables hold

// code word of a (plane, slope group): tap offsets (2 bits per slope), the
// window's first staged row (bits 8..15), per row group "window outside the
// volume" (bits 16..31)
constexpr int kCodeRowShift = 8;
constexpr int kCodeSkipShift = 16;

struct XshiftArgs {
    petl_geom G;
    int step;  // view step of the members' view ranges
    int NXc;   // scratch row pitch (columns, a multiple of 4)
    Tables T;
    Members M;  // volumes (in) and views of the chunk
};

constexpr int XZB = 8;      // volume rows z per k_xshift block
constexpr int XMAXNX = 1024;  // longest volume row k_xshift stages

// X rows of a chunk of views.  A block stages rows z0..z0+7 of plane y of
// one member's volume in shared memory once and writes them shifted for
// every view of that member in the chunk, one float4 of columns per thread
// and step.  Grid (ceil(NZ / 8), NY, members).
template <class TF, int NM>
__global__ void __launch_bounds__(256) k_xshift(float* __restrict__ X, const XshiftArgs A)
{
    __shared__ float rowbuf[XZB * XMAXNX];
    const petl_geom& G = A.G;
    const int NY = G.numY, NX = G.numX, NZ = G.numZ;
    const int y = blockIdx.y, z0 = blockIdx.x * XZB;
    const int b = NM == 1 ? 0 : int(blockIdx.z);
    const int nz = min(XZB, NZ - z0);
    const int nq = A.NXc >> 2;  // float4 columns per row
    const TF* __restrict__ f = static_cast<const TF*>(member_pick<NM>(A.M.in, b));
    for (int e = threadIdx.x; e < nz * NX; e += blockDim.x) {
        const int r = e / NX, x = e - r * NX;
        rowbuf[r * NX + x] = Store<TF>::ld(f[(size_t(z0 + r) * NY + y) * NX + x]);
    }
    __syncthreads();
    const int first = member_pick<NM>(A.M.first, b), nvb = member_pick<NM>(A.M.nv, b);
    for (int iv = 0; iv < nvb; iv++) {
        const Shift xs = A.T.xt[size_t(first + iv * A.step) * NY + y];
        const float w1 = xs.w, w0 = 1.0f - xs.w;
        float* Xv = X + (size_t(b * A.M.nvm + iv) * NY + y) * NZ * A.NXc;
        for (int e = threadIdx.x; e < nz * nq; e += blockDim.x) {
            const int r = e / nq, c = (e - r * nq) * 4;
            const float* fr = rowbuf + r * NX;
            float v[5];
#pragma unroll
            for (int i = 0; i < 5; i++) {
                const int ix = c + xs.d + i;
                v[i] = unsigned(ix) < unsigned(NX) ? fr[ix] : 0.0f;
            }
            const float4 o = make_float4(fmaf(w1, v[1], w0 * v[0]), fmaf(w1, v[2], w0 * v[1]),
                                         fmaf(w1, v[3], w0 * v[2]), fmaf(w1, v[4], w0 * v[3]));
            // streaming store: the scratch is read once, by the next kernel
            __stcs(reinterpret_cast<float4*>(Xv + size_t(z0 + r) * A.NXc + c), o);
        }
    }
}

struct ZsumArgs {
    petl_geom G;
    int step;      // view step of the members' view ranges
    int v1_first;  // first slope of the launch's slope blocks
    int v1_end;    // one past its last slope
    int sg;        // slope groups per CTA (4; 1 or 2 for a tail block of at most 8 slopes)
    int n_colblk;  // ceil(N_u0 / 64)
    int n_rowblk;  // ceil(N_u1 / rows per CTA)
    int nrb;       // staged rows per plane (rows per CTA + CTA shift spread + 1, bounded on the host)
    int ns;        // ring stages, two planes each
    int pstride;   // floats per staged plane (nrb + ZDMAX rows of 64; a multiple of 32)
    // shared-memory layout (byte offsets, set by the host): weights, codes,
    // live planes, barriers
    unsigned off_w, off_code, off_plane, off_bar;
    Tables T;
    int* err;
    unsigned wait_limit;  // bound of the waits on staged data (wait_limit(): kWaitLimit or 0)
    Members M;  // planograms (out), measured planograms (meas) and views of the chunk
};

// z taps of one slope: all first-tap FMAs, then all second-tap FMAs (16
// independent chains per pass)
template <int O>
__device__ __forceinline__ void zsum_taps(float2 (&acc)[ZK], const float2 (&W)[ZWN], float2 w0, float2 w1)
{
#pragma unroll
    for (int k = 0; k < ZK; k++) acc[k] = fma2(w0, W[k + O], acc[k]);
#pragma unroll
    for (int k = 0; k < ZK; k++) acc[k] = fma2(w1, W[k + O + 1], acc[k]);
}

// z taps of the four slopes of a warp with compile-time tap offsets
// (PC: 2 bits per slope), each slope's FMAs as zsum_taps orders them.
template <int PC>
__device__ __forceinline__ void zsum4(float2 (&acc)[ZV][ZK], const float2 (&W)[ZWN], const float (&wj)[ZV])
{
    zsum_taps<(PC >> 0) & 3>(acc[0], W, dup(1.0f - wj[0]), dup(wj[0]));
    zsum_taps<(PC >> 2) & 3>(acc[1], W, dup(1.0f - wj[1]), dup(wj[1]));
    zsum_taps<(PC >> 4) & 3>(acc[2], W, dup(1.0f - wj[2]), dup(wj[2]));
    zsum_taps<(PC >> 6) & 3>(acc[3], W, dup(1.0f - wj[3]), dup(wj[3]));
}

// TG: planogram storage (float or bfloat16); X and the arithmetic are FP32.
// Warp w: slope group w % sg, row group w / sg.  The copy of stage j is
// started by lane 0 of warp j % 16 once every warp has released the slot.
template <class TG, int NM>
__global__ void __launch_bounds__(ZNT, 1)
k_fwd_zsum(const __grid_constant__ CUtensorMap xmap, const ZsumArgs A)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sg = A.sg, rows = ZK * (ZWARPS / sg);
    const int gv = warp % sg, gr = warp / sg;
    const int vi = blockIdx.y;  // view slot within the chunk
    const int mb = NM == 1 ? 0 : vi / A.M.nvm, mv = vi - mb * A.M.nvm;
    if (mv >= member_pick<NM>(A.M.nv, mb)) return;  // a member with fewer views than the slots
    const int iv0 = member_pick<NM>(A.M.first, mb) + mv * A.step;
    TG* __restrict__ g = static_cast<TG*>(member_pick<NM>(A.M.out, mb));
    const TG* __restrict__ meas = static_cast<const TG*>(member_pick<NM>(A.M.meas, mb));
    int t = blockIdx.x;
    const int colblk = t % A.n_colblk;
    t /= A.n_colblk;
    const int rowblk = t % A.n_rowblk;
    t /= A.n_rowblk;
    const int v1a = A.v1_first + t * (ZV * sg);
    const int v1b = min(v1a + ZV * sg, A.v1_end) - 1;  // last slope of the CTA
    const int nsl = v1b - v1a + 1;
    const int cta_row0 = rowblk * rows, col0 = colblk * ZCOLS;
    const int jw = gv * ZV;              // first slope of this warp, relative to v1a
    const int row0 = cta_row0 + gr * ZK;  // first row of this warp
    const int NY = G.numY, NZ = G.numZ, NX = G.numX;
    const int ns = A.ns, npl = min(NY, ZMAXPLANES);

    float* ringp = reinterpret_cast<float*>(smem);                      // [ns][2][pstride]
    float4* s_w1 = reinterpret_cast<float4*>(smem + A.off_w);            // [npl][4]
    uint32_t* s_code = reinterpret_cast<uint32_t*>(smem + A.off_code);   // [npl][4]
    int2* s_plane = reinterpret_cast<int2*>(smem + A.off_plane);         // [npl] (y, first staged row)
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + A.off_bar);      // [ZNSMAX]
    uint64_t* empty = full + ZNSMAX;                                     // [ZNSMAX]
    int* s_n = reinterpret_cast<int*>(empty + ZNSMAX);
    volatile int* s_abort = s_n + 1;  // a consumer gave up a wait: start no further copies
    int* s_round = s_n + 2;           // [ZNSMAX] round of the copy last started in a slot

    // a tile outside the visible bins of every slope stays zero
    const int2 ub0 = A.T.ub0[iv0];
    bool any_row = false;
    for (int v1 = v1a; v1 <= v1b; v1++) {
        const int2 u = A.T.ub1[v1];
        any_row |= !(cta_row0 > u.y || cta_row0 + rows - 1 < u.x);
    }
    const bool live = any_row && !(col0 > ub0.y || col0 + ZCOLS - 1 < ub0.x);

    // slopes of this warp whose rows can be visible
    unsigned wmask = 0;
#pragma unroll
    for (int j = 0; j < ZV; j++) {
        if (jw + j < nsl) {
            const int2 u = A.T.ub1[v1a + jw + j];
            if (!(row0 > u.y || row0 + ZK - 1 < u.x)) wmask |= 1u << j;
        }
    }

    float2 acc[ZV][ZK];
#pragma unroll
    for (int j = 0; j < ZV; j++)
#pragma unroll
        for (int k = 0; k < ZK; k++) acc[j][k] = make_float2(0.0f, 0.0f);

    if (live) {  // CTA-uniform
        // planes whose staged window meets the volume, compacted in order
        if (warp == 0) {
            int n = 0;
            for (int yb = 0; yb < NY; yb += 32) {
                const int y = yb + lane;
                bool ok = false;
                int wlo = 0;
                if (y < NY) {
                    const Shift xs = A.T.xt[size_t(iv0) * NY + y];
                    const int da = A.T.zt[size_t(v1a) * NY + y].d, db = A.T.zt[size_t(v1b) * NY + y].d;
                    const int dzmin = min(da, db);
                    const int nr = rows + (max(da, db) - dzmin) + 1;
                    const int cx = col0 + xs.d;
                    wlo = cta_row0 + dzmin;
                    ok = !(cx + ZCOLS < 0 || cx >= NX || wlo + nr - 1 < 0 || wlo >= NZ);
                    if (ok && nr > A.nrb) {
                        atomicOr(A.err, kErrLayout);
                        ok = false;
                    }
                }
                const unsigned b = __ballot_sync(0xffffffffu, ok);
                const int idx = n + __popc(b & ((1u << lane) - 1u));
                if (ok && idx < npl) s_plane[idx] = make_int2(y, wlo);
                n += __popc(b);
            }
            if (lane == 0) {
                if (n > npl) {  // the host bounds numY; never index past the tables
                    atomicOr(A.err, kErrLayout);
                    n = npl;
                }
                s_n[0] = n;
                *s_abort = 0;
                for (int s = 0; s < ns; s++) {
                    mbar_init(&full[s], 1);
                    mbar_init(&empty[s], ZWARPS);
                    s_round[s] = -1;
                }
                fence_barrier_init();
            }
        }
        __syncthreads();
        const int nlive = s_n[0];

        // per (plane, slope group): window row, tap offsets, skip bits, weights
        for (int e = tid; e < nlive * sg; e += ZNT) {
            const int li = e / sg, q = e - li * sg;
            const int2 pl = s_plane[li];
            const int y = pl.x, wlo = pl.y;
            const int dzmin = wlo - cta_row0;
            int d[ZV];
            float w[ZV];
            int base = 1 << 30;
#pragma unroll
            for (int j = 0; j < ZV; j++) {
                d[j] = 0;
                w[j] = 0.0f;
                if (q * ZV + j < nsl) {
                    const Shift zs = A.T.zt[size_t(v1a + q * ZV + j) * NY + y];
                    d[j] = zs.d;
                    w[j] = zs.w;
                    base = min(base, zs.d);
                }
            }
            uint32_t code = 0xffffu << kCodeSkipShift;  // no slope in this group
            if (base != (1 << 30)) {
                const int xoff = base - dzmin;  // >= 0: the shifts are monotone in v1
                // the window of the last row group ends inside the plane's rows (nrb + ZDMAX)
                if (xoff < 0 || xoff + rows - ZK + ZWN > A.nrb + ZDMAX || xoff > 255) {
                    atomicOr(A.err, kErrLayout);
                } else {
                    code = uint32_t(xoff) << kCodeRowShift;
#pragma unroll
                    for (int j = 0; j < ZV; j++) {
                        if (q * ZV + j >= nsl) continue;
                        const int o = d[j] - base;
                        if (o > ZDMAX) atomicOr(A.err, kErrLayout);
                        code |= uint32_t(min(o, ZDMAX)) << (2 * j);
                    }
                    for (int r = 0; r < ZWARPS / sg; r++) {
                        const int iz0 = wlo + xoff + r * ZK;  // volume row of window row 0
                        if (iz0 + ZWN - 1 < 0 || iz0 >= NZ) code |= 1u << (kCodeSkipShift + r);
                    }
                }
            }
            s_code[li * 4 + q] = code;
            s_w1[li * 4 + q] = make_float4(w[0], w[1], w[2], w[3]);
        }
        __syncthreads();

        const int nst = (nlive + 1) / 2;  // ring stages of this CTA
        const uint32_t box_bytes = uint32_t(ZCOLS) * uint32_t(A.nrb) * 4u;
        bool dead = false;
        // stage j holds planes 2j and 2j + 1; it reuses its slot once every
        // warp has released stage j - ns
        auto issue = [&](int j) {
            const int slot = j % ns, round = j / ns;
            if (round > 0 && !mbar_wait(&empty[slot], uint32_t((round - 1) & 1), A.err, A.wait_limit)) return false;
            if (*s_abort) return false;
            fence_proxy_async_smem();
            const int np = min(2, nlive - 2 * j);
            mbar_arrive_expect_tx(&full[slot], box_bytes * uint32_t(np));
            for (int h = 0; h < np; h++) {
                const int2 pl = s_plane[2 * j + h];
                tma_load_4d(ringp + size_t(2 * slot + h) * A.pstride, &xmap, &full[slot], col0, pl.y, pl.x, vi);
            }
            s_round[slot] = round;
            return true;
        };
        if (tid == 0)
            for (int j = 0; j < ns - 1 && j < nst; j++) issue(j);
        // the next stage this warp starts: the first j >= ns - 1 with j % 16 == warp
        int my_next = warp + ZWARPS * ((ns - 1 - warp + ZWARPS - 1) / ZWARPS);
        if (my_next < ns - 1) my_next += ZWARPS;
        int slot = 0;
        uint32_t phase = 0;
        for (int j = 0; j < nst; j++) {
            if (j + ns - 1 == my_next) {
                if (lane == 0 && !dead && my_next < nst && !issue(my_next)) dead = true;
                my_next += ZWARPS;
            }
            if (!dead) dead = !mbar_wait(&full[slot], phase, A.err, A.wait_limit);
            if (dead) *s_abort = 1;  // before this warp releases the slot
#pragma unroll 1
            for (int h = 0; h < 2 && !dead; h++) {
                const int li = 2 * j + h;
                if (li >= nlive) break;
                const uint32_t code = s_code[li * 4 + gv];
                if (!wmask || ((code >> (kCodeSkipShift + gr)) & 1u)) continue;
                const float4 w1 = s_w1[li * 4 + gv];
                const float wj[ZV] = {w1.x, w1.y, w1.z, w1.w};
                const float* Xr = ringp + size_t(2 * slot + h) * A.pstride +
                                  (int((code >> kCodeRowShift) & 0xffu) + gr * ZK) * ZCOLS + 2 * lane;
                float2 W[ZWN];
#pragma unroll
                for (int i = 0; i < ZWN; i++) W[i] = *reinterpret_cast<const float2*>(Xr + i * ZCOLS);
                // the offsets of four consecutive slopes move by at most one
                // row per slope: one dispatch over the 15 monotone patterns
                bool done = wmask == 0xFu;
                if (done) {
                    switch (code & 0xffu) {
                        case 0x00: zsum4<0x00>(acc, W, wj); break;
                        case 0x40: zsum4<0x40>(acc, W, wj); break;
                        case 0x50: zsum4<0x50>(acc, W, wj); break;
                        case 0x90: zsum4<0x90>(acc, W, wj); break;
                        case 0x54: zsum4<0x54>(acc, W, wj); break;
                        case 0x94: zsum4<0x94>(acc, W, wj); break;
                        case 0xA4: zsum4<0xA4>(acc, W, wj); break;
                        case 0xE4: zsum4<0xE4>(acc, W, wj); break;
                        case 0x01: zsum4<0x01>(acc, W, wj); break;
                        case 0x05: zsum4<0x05>(acc, W, wj); break;
                        case 0x15: zsum4<0x15>(acc, W, wj); break;
                        case 0x06: zsum4<0x06>(acc, W, wj); break;
                        case 0x16: zsum4<0x16>(acc, W, wj); break;
                        case 0x1A: zsum4<0x1A>(acc, W, wj); break;
                        case 0x1B: zsum4<0x1B>(acc, W, wj); break;
                        default: done = false;
                    }
                }
                if (!done) {
#pragma unroll
                    for (int jj = 0; jj < ZV; jj++) {
                        if (!((wmask >> jj) & 1u)) continue;
                        const float2 a1 = dup(wj[jj]), a0 = dup(1.0f - wj[jj]);
                        switch ((code >> (2 * jj)) & 3u) {
                            case 0: zsum_taps<0>(acc[jj], W, a0, a1); break;
                            case 1: zsum_taps<1>(acc[jj], W, a0, a1); break;
                            case 2: zsum_taps<2>(acc[jj], W, a0, a1); break;
                            default: zsum_taps<3>(acc[jj], W, a0, a1); break;
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot]);
            if (++slot == ns) {
                slot = 0;
                phase ^= 1u;
            }
        }
        if (__syncthreads_or(dead)) {
            // a wait gave up: drain the copies still in flight, write nothing
            if (tid == 0)
                for (int s = 0; s < ns; s++)
                    if (s_round[s] >= 0) mbar_wait(&full[s], uint32_t(s_round[s] & 1), nullptr);
            return;
        }
    }

    // epilogue: scale, ray masks, optional MLEM ratio
    const int colA = col0 + 2 * lane;
    const bool pairs = (G.N_u0 & 1) == 0;  // float2 accesses stay 8-byte aligned
#pragma unroll
    for (int j = 0; j < ZV; j++) {
        const int v1 = v1a + jw + j;
        if (jw + j >= nsl) continue;
        const float S = A.T.S[size_t(v1) * G.N_v0 + iv0];
        const int2 u1r = A.T.ub1[v1];
#pragma unroll
        for (int k = 0; k < ZK; k++) {
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

// Scratch budget of the x-shift pass (bytes of FP32 X per chunk of views);
// PETL_SPLIT_SCRATCH_MB overrides it.

// Launch layout of k_fwd_zsum for one range of slope blocks.
struct ZsumLaunch {
    ZsumArgs A;
    CUtensorMap map;
    size_t smem;
    unsigned nblk;  // CTAs per view
};

// Layout of the blocks of slopes [v1_first, v1_end) with sg slope groups per
// CTA: false when it breaks a layout rule.
bool zsum_layout(const petl_geom& G, const ViewRange& vr, int v1_first, int v1_end, int sg, double step,
                 const float* X, int NXc, int nv, const Tables& T, int* err, ZsumLaunch& L)
{
    const int rows = ZK * (ZWARPS / sg);
    const int nrb = rows + shift_spread(ZV * sg - 1, step) + 1;
    if (nrb > 256 - ZDMAX) return false;  // TMA box rows; the window row fits 8 bits
    ZsumArgs& A = L.A;
    A = ZsumArgs{};
    A.G = G;
    A.step = vr.iv0_step;
    A.v1_first = v1_first;
    A.v1_end = v1_end;
    A.sg = sg;
    A.n_colblk = int(ceil_div(G.N_u0, ZCOLS));
    A.n_rowblk = int(ceil_div(G.N_u1, rows));
    A.nrb = nrb;
    A.pstride = ((nrb + ZDMAX) * ZCOLS + 31) & ~31;  // 128-byte aligned planes
    A.T = T;
    A.err = err;
    A.wait_limit = wait_limit();
    // shared memory: the ring, then the per-CTA tables and the barriers
    const size_t np = size_t(std::min(G.numY, ZMAXPLANES));
    const size_t b_w = np * 4 * sizeof(float4), b_code = np * 4 * 4, b_plane = np * 8;
    const size_t b_bar = 2 * ZNSMAX * 8 + (2 + ZNSMAX) * 4;
    auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
    const size_t fixed = al(b_w) + al(b_code) + al(b_plane) + al(b_bar);
    const size_t stage = size_t(2) * A.pstride * 4;
    A.ns = int(std::min<size_t>(ZNSMAX, (227 * 1024 - std::min<size_t>(fixed, 227 * 1024)) / stage));
    if (A.ns < 2) return false;
    const size_t ring = size_t(A.ns) * stage;
    A.off_w = unsigned(ring);
    A.off_code = unsigned(A.off_w + al(b_w));
    A.off_plane = unsigned(A.off_code + al(b_code));
    A.off_bar = unsigned(A.off_plane + al(b_plane));
    L.smem = A.off_bar + al(b_bar);
    if (L.smem > 227 * 1024) return false;
    L.nblk = unsigned(A.n_colblk) * unsigned(A.n_rowblk) * ceil_div(v1_end - v1_first, ZV * sg);
    const uint64_t dims[4] = {uint64_t(NXc), uint64_t(G.numZ), uint64_t(G.numY), uint64_t(nv)};
    const uint64_t strides[3] = {uint64_t(NXc) * 4, uint64_t(NXc) * G.numZ * 4, uint64_t(NXc) * G.numZ * G.numY * 4};
    const uint32_t box[4] = {uint32_t(ZCOLS), uint32_t(nrb), 1u, 1u};
    return encode_tensor_map(&L.map, X, 4, dims, strides, box, 4);
}

}  // namespace

size_t split_scratch_budget()
{
    static const long long env_mb = [] {
        const char* e = std::getenv("PETL_SPLIT_SCRATCH_MB");
        return e ? std::atoll(e) : 0LL;
    }();
    if (env_mb > 0) return size_t(env_mb) << 20;
    // the device's memory size, looked up once per device (a query per call
    // would cost host time on the launch path)
    static std::mutex mu;
    static size_t total[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return size_t(1) << 30;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!total[dev]) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
            cudaGetLastError();
            return size_t(1) << 30;
        }
        total[dev] = prop.totalGlobalMem;
    }
    return std::min(size_t(5) << 30, total[dev] / 8);
}

// Forward projection of the members' views.  One member: its views in
// chunks of at most the scratch budget (and chunk_cap); several: one chunk,
// else kNotApplicable.
template <class TF, class TG>
int project_split_m(const petl_geom& G, const Members& M0, const ViewRange& vr, const Tables& T, cudaStream_t st,
                    int chunk_cap, const ChunkHook* hook)
{
    const int nb = M0.nb;
    if (nb < 1 || nb > kMaxMembers) return kNotApplicable;
    int nvmax = 0;
    for (int b = 0; b < nb; b++) nvmax = std::max(nvmax, M0.nv[b]);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (nvmax <= 0 || nv1 <= 0) return 0;
    // the x pass writes a volume per view whatever the slope count: below
    // about ten slopes the single-pass kernel is cheaper than that round trip
    if (nv1 < kSplitMinSlopes) return kNotApplicable;
    if (G.numY > ZMAXPLANES || G.numZ > 65535 * 4) return kNotApplicable;
    const double step = double(G.T_v1) * plane_ymax(G) / double(G.T_z);  // shift change per slope
    if (shift_spread(ZV - 1, step) > ZDMAX) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;

    // chunks of views whose X fits the scratch budget, balanced in size
    const int NXc = (G.N_u0 + 3) & ~3;
    const size_t per_view = size_t(G.numY) * G.numZ * NXc * 4;
    if (G.numX > XMAXNX || G.numY > 65535) return kNotApplicable;  // k_xshift row buffer, grid.y
    const size_t fit = std::max<size_t>(1, split_scratch_budget() / per_view);
    int nv, nchunks;
    if (nb == 1) {
        nv = int(std::min<size_t>(size_t(nvmax), fit));
        if (chunk_cap > 0) nv = std::min(nv, chunk_cap);
        nchunks = (nvmax + nv - 1) / nv;
        nv = (nvmax + nchunks - 1) / nchunks;
    } else {
        if (size_t(nb) * nvmax > fit || size_t(nb) * nvmax > 65535 || chunk_cap > 0) return kNotApplicable;
        nv = nvmax;
        nchunks = 1;
    }

    float* X = nullptr;
    if (scratch_alloc(reinterpret_cast<void**>(&X), per_view * nv * nb, st) != cudaSuccess) {
        cudaGetLastError();  // out of memory is not sticky: the caller takes the fused kernel
        return kNotApplicable;
    }
    // full blocks of 16 slopes; a tail of at most 8 slopes takes CTAs of 1 or
    // 2 slope groups over 128 or 64 rows instead of a mostly idle full block
    const int ntail = nv1 % ZSL;
    const int tail_sg = ntail == 0 ? 0 : ntail <= ZV ? 1 : ntail <= 2 * ZV ? 2 : 0;
    const int v1_split = vr.iv1_end - (tail_sg ? ntail : 0);
    ZsumLaunch L[2];
    int nl = 0;
    bool ok = true;
    if (v1_split > vr.iv1_begin)
        ok = zsum_layout(G, vr, vr.iv1_begin, v1_split, ZSG, step, X, NXc, nv * nb, T, err, L[nl++]);
    if (ok && tail_sg) ok = zsum_layout(G, vr, v1_split, vr.iv1_end, tail_sg, step, X, NXc, nv * nb, T, err, L[nl++]);
    if (!ok) {
        cudaFreeAsync(X, st);
        return kNotApplicable;
    }
    // kernels compiled for one member where there is one
    auto kz = nb == 1 ? k_fwd_zsum<TG, 1> : k_fwd_zsum<TG, kMaxMembers>;
    auto kx = nb == 1 ? k_xshift<TF, 1> : k_xshift<TF, kMaxMembers>;
    size_t smem_max = 0;
    for (int l = 0; l < nl; l++) smem_max = std::max(smem_max, L[l].smem);
    cudaError_t e = cudaFuncSetAttribute(kz, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_max));
    for (int c = 0; c < nchunks && e == cudaSuccess; c++) {
        Members M = M0;
        const int vi0 = c * nv;
        int nvc = nv;
        if (nb == 1) {
            nvc = std::min(nv, nvmax - vi0);
            M.first[0] = M0.first[0] + vi0 * vr.iv0_step;
            M.nv[0] = nvc;
        }
        M.nvm = nvc;
        XshiftArgs XA{G, vr.iv0_step, NXc, T, M};
        kx<<<dim3(ceil_div(G.numZ, XZB), unsigned(G.numY), unsigned(nb)), 256, 0, st>>>(X, XA);
        note_launch();
        for (int l = 0; l < nl; l++) {
            L[l].A.M = M;
            kz<<<dim3(L[l].nblk, unsigned(nvc * nb)), ZNT, L[l].smem, st>>>(L[l].map, L[l].A);
            note_launch();
        }
        e = cudaGetLastError();
        if (e == cudaSuccess && hook && hook->fn) hook->fn(hook->ctx, vi0, nvc);
    }
    cudaFreeAsync(X, st);
    if (e != cudaSuccess) {
        set_error(std::string("project_split: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

template <class TF, class TG>
int project_split_t(const petl_geom& G, const TF* f, TG* g, const ViewRange& vr, const TG* meas, const Tables& T,
                    cudaStream_t st, int chunk_cap, const ChunkHook* hook)
{
    Members M;
    M.nb = 1;
    M.first[0] = vr.iv0_first;
    M.nv[0] = vr.n_v0(G.N_v0);
    M.in[0] = f;
    M.out[0] = g;
    M.meas[0] = meas;
    if (M.nv[0] <= 0 || vr.iv1_end <= vr.iv1_begin) return 0;
    return project_split_m<TF, TG>(G, M, vr, T, st, chunk_cap, hook);
}

int project_split(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                  const Tables& T, cudaStream_t st, int chunk_cap, const ChunkHook* hook)
{
    return project_split_t<float, float>(G, f, g, vr, meas, T, st, chunk_cap, hook);
}

int project_split_bf16(const petl_geom& G, const __nv_bfloat16* f, __nv_bfloat16* g, const ViewRange& vr,
                       const __nv_bfloat16* meas, const Tables& T, cudaStream_t st)
{
    return project_split_t<__nv_bfloat16, __nv_bfloat16>(G, f, g, vr, meas, T, st, 0, nullptr);
}

int project_split_members(const petl_geom& G, const Members& M, const ViewRange& vr, const Tables& T,
                          cudaStream_t st)
{
    return project_split_m<float, float>(G, M, vr, T, st, 0, nullptr);
}

}  // namespace shear
}  // namespace petl
