// Split backprojector (psi = 0, voxel pitch equal to the bin pitch): the
// transpose of the split forward (projector_split.cu), in the gather form of
// k_bwd_tma (projector_shear_tma.cu) for the reference semantics of
// src/projectors.cu:240-377 and for the exact adjoint.
//
// The voxel (x, y, z) receives, from view v0 and slope v1 on plane y,
//   S (1 - wz) g[v1][v0][z - dz][x - dx] + S wz g[v1][v0][z - dz - 1][x - dx]
// interpolated in x by (1 - wx, wx) over columns x - dx and x - dx - 1.  The
// two interpolations are separate kernels:
//
// * k_bwd_zgather sums the z taps over the slopes of one view into FP32
//   scratch B[view][y][z][c] (c = planogram column).  CTA = views of a group x
//   16 planes x 32 rows x 64 columns, 16 warps of 4 planes x 8 rows x 2
//   columns per lane; per slope the planogram rows the tile needs arrive by a
//   tiled TMA copy (no multicast) into a ring of two-slope stages with
//   full/empty mbarriers and a rotating copy issuer; window offsets, modes,
//   masks and weights are tabulated once per CTA.
// * k_bwd_xgather applies the x taps and sums the views of a chunk into the
//   volume (or an FP32 partial sum between chunks).
//
// Both do the float operations of k_bwd_tma in the same order (per voxel:
// z taps over the live slopes in ascending v1, tap 0 then tap 1; x taps over
// the views in order; the scale last), so the two paths agree bit for bit.
// As in the forward, a launch serves one call or up to kMaxMembers requests
// of one geometry (one tensor map per member's planogram).  A single slope
// at v1 = 0 (the rebinned planogram of FBP) takes k_bwd_zflat: its z sums
// do not depend on the plane.
// Every wait is bounded: a wait that gives up sets the device error word, the
// CTA drains its copies in flight and returns without writing.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {
namespace shear {

namespace {

constexpr int GP = 4;               // planes per warp
constexpr int GK = 8;               // rows per warp
constexpr int GPG = 4;              // plane groups per CTA
constexpr int GRG = 4;              // row groups per CTA
constexpr int GPL = GP * GPG;       // planes per CTA
constexpr int GROWS = GK * GRG;     // rows per CTA
constexpr int GCOLS = 64;           // columns per CTA, two per lane
constexpr int GWARPS = GPG * GRG;
constexpr int GNT = 32 * GWARPS;
constexpr int GDW = 2;              // largest shift difference among a warp's planes
constexpr int GWN = GK + GDW + 1;   // register window rows
// ring stages: two (of two slopes each) measured fastest; deeper rings
// (3-8 stages) ran 3-10 % slower at the 256x256x128 workload
constexpr int GNSMAX = 2;
constexpr int GV1MAX = 128;         // slopes per call at most
constexpr int GVG = 4;              // views per CTA at most
constexpr int kPatGen = 15;         // no straight-line pattern: per-plane taps

// Window offsets of a plane group's 4 planes when all are fully visible and
// their shifts differ by at most one row: o0 | o1 << 2 | o2 << 4 | o3 << 6.
constexpr int kNumPat = 7;
__host__ __device__ constexpr int gpat_offsets(int pid)
{
    return pid == 0 ? 0x00 : pid == 1 ? 0x40 : pid == 2 ? 0x50 : pid == 3 ? 0x54
         : pid == 4 ? 0x01 : pid == 5 ? 0x05 : 0x15;
}

// Entry of a (slope, warp).  code: plane modes and offsets (4 bits per
// plane: mode 0 none / 1 full / 2 masked rows, offset << 2), path << 16
// (0..6: the straight-line pattern of fully visible planes; 8..14: the same
// pattern with per-plane row intervals; kPatGen: per-plane taps), window row
// in the stage << 20.  vm: window rows holding visible bins (adjoint).  ivl:
// per plane (8 bits each) the mask of output rows that receive the slope:
// the rows inside the visible range (adjoint: all) or passing the voxel
// test (reference).
struct __align__(16) GEntry {
    uint32_t code;
    uint32_t vm;
    uint32_t ivl;
    uint32_t pad;
};

struct ZgatherArgs {
    petl_geom G;
    ViewRange vr;  // slopes and view step (the members hold their views)
    int vg;        // views per CTA
    int gpm;       // CTAs along y per member: ceil(view slots per member / vg)
    int n_colblk;  // ceil(N_u0 / 64)
    int n_rowblk;  // ceil(numZ / 32)
    int brb;       // staged planogram rows per slope (33 + CTA shift spread, bounded on the host)
    int ns;        // ring stages, two slopes each
    int sstride;   // elements per staged slope (brb + 2 rows of 64; 128-byte multiple)
    int NUc;       // scratch row pitch (columns)
    int v1cap;     // slopes the per-CTA tables hold (the call's slope count)
    Tables T;
    int* err;
    unsigned wait_limit;  // bound of the waits on staged data (wait_limit(): kWaitLimit or 0)
    Members M;  // views of the chunk per member (the planograms are the tensor maps)
};

// tensor maps of the members' planograms
template <int NM>
struct GMaps {
    CUtensorMap m[NM];
};

// z taps of one plane (two columns): Z[k] += w0 W[O + k + 1] then w1 W[O + k],
// with per-row 0/1 masks when MASK (vm: window rows, om: output rows).
template <int O, bool MASK>
__device__ __forceinline__ void g_taps(float2 (&Z)[GK], const float2 (&W)[GWN], float w0, float w1, uint32_t vm,
                                       uint32_t om)
{
    if (MASK) {
#pragma unroll
        for (int k = 0; k < GK; k++) {
            const bool kb = (vm >> (O + k + 1)) & (om >> k) & 1u, ka = (vm >> (O + k)) & (om >> k) & 1u;
            const float2 b = kb ? W[O + k + 1] : make_float2(0.0f, 0.0f);
            const float2 a = ka ? W[O + k] : make_float2(0.0f, 0.0f);
            Z[k] = make_float2(fmaf(w1, a.x, fmaf(w0, b.x, Z[k].x)), fmaf(w1, a.y, fmaf(w0, b.y, Z[k].y)));
        }
    } else {
        const float2 a0 = dup(w0), a1 = dup(w1);
#pragma unroll
        for (int k = 0; k < GK; k++) Z[k] = fma2(a0, W[O + k + 1], Z[k]);
#pragma unroll
        for (int k = 0; k < GK; k++) Z[k] = fma2(a1, W[O + k], Z[k]);
    }
}

template <int PID>
__device__ __forceinline__ void g_taps4(float2 (&Z)[GP][GK], const float2 (&W)[GWN], float4 wa, float4 wb)
{
    constexpr int o = gpat_offsets(PID);
    g_taps<(o >> 0) & 3, false>(Z[0], W, wa.x, wa.y, 0u, 0u);
    g_taps<(o >> 2) & 3, false>(Z[1], W, wa.z, wa.w, 0u, 0u);
    g_taps<(o >> 4) & 3, false>(Z[2], W, wb.x, wb.y, 0u, 0u);
    g_taps<(o >> 6) & 3, false>(Z[3], W, wb.z, wb.w, 0u, 0u);
}

// z taps of one plane restricted to the output rows of mask m (predicated;
// rows outside receive nothing, as the masked taps' zero operands give)
template <int O>
__device__ __forceinline__ void g_taps_ivl(float2 (&Z)[GK], const float2 (&W)[GWN], float w0, float w1,
                                           uint32_t m)
{
    const float2 a0 = dup(w0), a1 = dup(w1);
#pragma unroll
    for (int k = 0; k < GK; k++)
        if ((m >> k) & 1u) Z[k] = fma2(a0, W[O + k + 1], Z[k]);
#pragma unroll
    for (int k = 0; k < GK; k++)
        if ((m >> k) & 1u) Z[k] = fma2(a1, W[O + k], Z[k]);
}

template <int PID>
__device__ __forceinline__ void g_taps4_ivl(float2 (&Z)[GP][GK], const float2 (&W)[GWN], float4 wa, float4 wb,
                                            uint32_t ivl)
{
    constexpr int o = gpat_offsets(PID);
    g_taps_ivl<(o >> 0) & 3>(Z[0], W, wa.x, wa.y, ivl);
    g_taps_ivl<(o >> 2) & 3>(Z[1], W, wa.z, wa.w, ivl >> 8);
    g_taps_ivl<(o >> 4) & 3>(Z[2], W, wb.x, wb.y, ivl >> 16);
    g_taps_ivl<(o >> 6) & 3>(Z[3], W, wb.z, wb.w, ivl >> 24);
}

// TG: planogram storage (float or bfloat16); B and the arithmetic are FP32.
// Warp w: plane group w % 4, row group w / 4.
template <bool ADJ, class TG, int NM>
__global__ void __launch_bounds__(GNT, 1)
k_bwd_zgather(const __grid_constant__ GMaps<NM> gmaps, float* __restrict__ B, const ZgatherArgs A)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = warp % GPG, r = warp / GPG;
    int t = blockIdx.x;
    const int colblk = t % A.n_colblk;
    t /= A.n_colblk;
    const int rowblk = t % A.n_rowblk;
    const int plblk = t / A.n_rowblk;
    const int p0 = plblk * GPL, r0 = rowblk * GROWS, col0 = colblk * GCOLS;
    const int z0 = r0 + r * GK;  // first row of this warp
    const int mb = NM == 1 ? 0 : blockIdx.y / A.gpm;  // member
    const int vfirst = (blockIdx.y - mb * A.gpm) * A.vg;  // first view of this CTA in the member's chunk
    const int nvw = min(A.vg, member_pick<NM>(A.M.nv, mb) - vfirst);  // views of this CTA
    if (nvw <= 0) return;  // a member with fewer views than the slots
    const int vbase = member_pick<NM>(A.M.first, mb) + vfirst * A.vr.iv0_step;  // view of k = 0
    const int sbase = mb * A.M.nvm + vfirst;                                // its scratch slot
    const CUtensorMap* gmap = &gmaps.m[0];
#pragma unroll
    for (int i = 1; i < NM; i++)
        if (mb == i) gmap = &gmaps.m[i];
    const int NY = G.numY, NZ = G.numZ, NU1 = G.N_u1;
    const int ns = A.ns;

    TG* ringp = reinterpret_cast<TG*>(smem);                                           // [ns][2][sstride]
    const int vcap = A.v1cap;
    GEntry* s_ent = reinterpret_cast<GEntry*>(smem + size_t(ns) * 2 * A.sstride * sizeof(TG));  // [vcap][16]
    float2* s_wt = reinterpret_cast<float2*>(s_ent + vcap * GWARPS);                    // [vg][vcap][16]
    int2* s_sl = reinterpret_cast<int2*>(s_wt + size_t(A.vg) * vcap * GPL);             // (v1, first staged row)
    uint64_t* full = reinterpret_cast<uint64_t*>(s_sl + vcap);                          // [GNSMAX]
    uint64_t* empty = full + GNSMAX;                                                    // [GNSMAX]
    int* s_n = reinterpret_cast<int*>(empty + GNSMAX);
    volatile int* s_abort = s_n + 1;
    int* s_round = s_n + 2;  // [GNSMAX]

    // ---- slopes whose rows reach the tile (warp 0), compacted in order
    if (warp == 0) {
        int n = 0;
        for (int vb = A.vr.iv1_begin; vb < A.vr.iv1_end; vb += 32) {
            const int v1 = vb + lane;
            bool ok = false;
            int grow = 0;
            if (v1 < A.vr.iv1_end) {
                int dmin = 1 << 30, dmax = -(1 << 30);
                for (int p = 0; p < GPL && p0 + p < NY; p++) {
                    const int d = A.T.zt[size_t(v1) * NY + p0 + p].d;
                    dmin = min(dmin, d);
                    dmax = max(dmax, d);
                }
                grow = r0 - dmax - 1;
                const int2 ub1 = A.T.ub1[v1];
                for (int p = 0; p < GPL && p0 + p < NY && !ok; p++) {
                    const int d = A.T.zt[size_t(v1) * NY + p0 + p].d;
                    // rows of the CTA that can receive this slope on plane p
                    const int lo = r0 - d - 1, hi = r0 + GROWS - 1 - d;
                    if (hi < 0 || lo >= NU1) continue;
                    if (ADJ) {
                        ok = !(hi < ub1.x || lo > ub1.y);
                    } else {
                        const int2 zv = A.T.zvis[size_t(v1) * NY + p0 + p];
                        ok = !(r0 + GROWS - 1 < zv.x || r0 > zv.y);
                    }
                }
                if (ok && dmax - dmin > A.brb - (GROWS + 1)) {
                    atomicOr(A.err, kErrLayout);
                    ok = false;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            const int idx = n + __popc(bal & ((1u << lane) - 1u));
            if (ok && idx < vcap) s_sl[idx] = make_int2(v1, grow);
            n += __popc(bal);
        }
        if (lane == 0) {
            if (n > vcap) {  // the host sizes the tables; never index past them
                atomicOr(A.err, kErrLayout);
                n = vcap;
            }
            s_n[0] = n;
            *s_abort = 0;
            for (int s = 0; s < ns; s++) {
                mbar_init(&full[s], 1);
                mbar_init(&empty[s], GWARPS);
                s_round[s] = -1;
            }
            fence_barrier_init();
        }
    }
    __syncthreads();
    const int nlive = s_n[0];

    // ---- per (slope, warp): plane modes, window offsets, pattern, masks
    for (int e = tid; e < nlive * GWARPS; e += GNT) {
        const int li = e / GWARPS, w = e - li * GWARPS;
        const int wq = w % GPG, wr = w / GPG;
        const int2 sl = s_sl[li];
        const int v1 = sl.x, grow = sl.y;
        const int zr = r0 + wr * GK;  // first row of warp w
        const int2 ub1 = A.T.ub1[v1];
        int dz[GP], mode[GP];
        int2 zv[GP];
        int dmx = -(1 << 30);
#pragma unroll
        for (int u = 0; u < GP; u++) {
            const int y = p0 + wq * GP + u;
            dz[u] = 0;
            mode[u] = 0;
            zv[u] = make_int2(0, -1);
            if (y >= NY) continue;
            dz[u] = A.T.zt[size_t(v1) * NY + y].d;
            const int lo = zr - dz[u] - 1, hi = zr + GK - 1 - dz[u];  // g rows touched
            if (hi < 0 || lo >= NU1) continue;
            if (ADJ) {
                if (hi < ub1.x || lo > ub1.y) continue;
                mode[u] = (lo >= ub1.x && hi <= ub1.y) ? 1 : 2;
            } else {
                zv[u] = A.T.zvis[size_t(v1) * NY + y];
                if (zr + GK - 1 < zv[u].x || zr > zv[u].y) continue;
                mode[u] = (zr >= zv[u].x && zr + GK - 1 <= zv[u].y) ? 1 : 2;
            }
            dmx = max(dmx, dz[u]);
        }
        GEntry en{0u, 0u, 0u, 0u};
        if (dmx != -(1 << 30)) {
            const int wfirst = zr - dmx - 1;  // g row of window row 0
            const int wrow = wfirst - grow;   // its row in the stage
            bool bad = wrow < 0 || wrow + GWN > A.brb + 2;
            uint32_t code = 0, ivl = 0, vm = 0;
            bool allfull = true;
            int offs = 0, olast = -1;
            for (int i = 0; i < GWN; i++)
                if (wfirst + i >= ub1.x && wfirst + i <= ub1.y) vm |= 1u << i;
#pragma unroll
            for (int u = 0; u < GP; u++) {
                const int o = dmx - dz[u];
                uint32_t iv = 0u;  // no rows
                if (mode[u]) {
                    if (o > GDW) bad = true;
                    code |= uint32_t(mode[u] | (min(o, 3) << 2)) << (4 * u);
                    if (ADJ || mode[u] == 1) {
                        iv = 0xffu;  // rows 0..7 (adjoint: invisible window rows are zeroed instead)
                    } else {
                        const int ka = max(zv[u].x - zr, 0), kb = min(zv[u].y - zr, GK - 1);
                        iv = kb >= ka ? (0xffu >> (7 - kb)) & (0xffu << ka) & 0xffu : 0u;
                    }
                }
                ivl |= iv << (8 * u);
                allfull = allfull && mode[u] == 1;
                // planes that receive nothing take a neighbour's offset
                // (monotone), so that a pattern can cover the group
                const int oe = mode[u] ? o : (olast >= 0 ? olast : dmx - dz[u]);
                if (mode[u]) olast = o;
                offs |= (min(oe, 3) & 3) << (2 * u);
            }
            // leading planes without rows: the offset of the first active one
            if (!mode[0]) {
                int ofirst = 0;
                for (int u = GP - 1; u >= 0; u--)
                    if (mode[u]) ofirst = dmx - dz[u];
                for (int u = 0; u < GP && !mode[u]; u++) offs = (offs & ~(3 << (2 * u))) | ((ofirst & 3) << (2 * u));
            }
            int pid = kPatGen;
            for (int c = 0; c < kNumPat; c++)
                if (gpat_offsets(c) == offs) pid = allfull ? c : c + 8;
            if (bad) {
                atomicOr(A.err, kErrLayout);
            } else {
                en.code = code | uint32_t(pid) << 16 | uint32_t(wrow) << 20;
                en.vm = vm;
                en.ivl = ivl;
            }
        }
        s_ent[li * GWARPS + w] = en;
    }
    // ---- weights (S (1 - w), S w) per view, slope and plane
    for (int e = tid; e < nvw * nlive * GPL; e += GNT) {
        const int k = e / (nlive * GPL), rem = e - k * (nlive * GPL);
        const int li = rem / GPL, p = rem - li * GPL;
        const int v1 = s_sl[li].x;
        const int v0 = vbase + k * A.vr.iv0_step;
        const int y = min(p0 + p, NY - 1);
        const float S = A.T.S[size_t(v1) * G.N_v0 + v0];
        const float w = A.T.zt[size_t(v1) * NY + y].w;
        s_wt[(k * vcap + li) * GPL + p] = make_float2(S * (1.0f - w), S * w);
    }
    __syncthreads();

    // ---- the ring: stage j holds slopes 2p and 2p + 1 (p = j mod nsp) of view j / nsp
    const int nsp = (nlive + 1) / 2;
    const int nst = nvw * nsp;
    const uint32_t box_bytes = uint32_t(GCOLS) * uint32_t(A.brb) * uint32_t(sizeof(TG));
    bool dead = false;
    // stage j reuses its slot once every warp has released stage j - ns
    auto issue = [&](int j) {
        const int slot = j % ns, round = j / ns;
        if (round > 0 && !mbar_wait(&empty[slot], uint32_t((round - 1) & 1), A.err, A.wait_limit)) return false;
        if (*s_abort) return false;
        fence_proxy_async_smem();
        const int k = j / nsp, pr = j - k * nsp;
        const int v0 = vbase + k * A.vr.iv0_step;
        const int np = min(2, nlive - 2 * pr);
        mbar_arrive_expect_tx(&full[slot], box_bytes * uint32_t(np));
        for (int h = 0; h < np; h++) {
            const int2 sl = s_sl[2 * pr + h];
            tma_load_4d(ringp + size_t(2 * slot + h) * A.sstride, gmap, &full[slot], col0, sl.y, v0, sl.x);
        }
        s_round[slot] = round;
        return true;
    };
    if (tid == 0)
        for (int j = 0; j < ns - 1 && j < nst; j++) issue(j);
    // the next stage this warp starts: the first j >= ns - 1 with j % 16 == warp
    int my_next = warp + GWARPS * ((ns - 1 - warp + GWARPS - 1) / GWARPS);
    if (my_next < ns - 1) my_next += GWARPS;

    float2 Z[GP][GK];
#pragma unroll
    for (int u = 0; u < GP; u++)
#pragma unroll
        for (int k = 0; k < GK; k++) Z[u][k] = make_float2(0.0f, 0.0f);

    // the z sums of view k go to the scratch (columns outside the view's
    // visible u0 range zeroed for the adjoint) and restart from zero
    auto store_view = [&](int k) {
        const int vi = sbase + k;  // scratch slot
        const int v0 = vbase + k * A.vr.iv0_step;
        const int2 u0r = ADJ ? A.T.ub0[v0] : make_int2(0, G.N_u0 - 1);
        const int c = col0 + 2 * lane;
        const bool vx = c >= u0r.x && c <= u0r.y, vy = c + 1 >= u0r.x && c + 1 <= u0r.y;
#pragma unroll
        for (int u = 0; u < GP; u++) {
            const int y = p0 + q * GP + u;
#pragma unroll
            for (int kk = 0; kk < GK; kk++) {
                const int z = z0 + kk;
                if (y < NY && z < NZ && c < G.N_u0) {
                    float* dst = B + ((size_t(vi) * NY + y) * NZ + z) * A.NUc + c;
                    const float2 v = make_float2(vx ? Z[u][kk].x : 0.0f, vy ? Z[u][kk].y : 0.0f);
                    if (c + 1 < G.N_u0)
                        __stcs(reinterpret_cast<float2*>(dst), v);
                    else
                        dst[0] = v.x;
                }
                Z[u][kk] = make_float2(0.0f, 0.0f);
            }
        }
    };

    int slot = 0;
    uint32_t phase = 0;
    int k = 0, pr = 0;  // view and slope pair of stage j
    for (int j = 0; j < nst; j++) {
        if (j + ns - 1 == my_next) {
            if (lane == 0 && !dead && my_next < nst && !issue(my_next)) dead = true;
            my_next += GWARPS;
        }
        // the hot wait keeps the compile-time bound (a run-time bound here
        // measured 1 % slower); the forced give-up reaches this kernel through
        // the slot waits of issue(), and the warps waiting here for a copy
        // that was then never started leave on the abort flag
        if (!dead) dead = !mbar_wait_abortable(&full[slot], phase, A.err, s_abort);
        if (dead) *s_abort = 1;  // before this warp releases the slot
#pragma unroll 1
        for (int h = 0; h < 2 && !dead; h++) {
            const int li = 2 * pr + h;
            if (li >= nlive) break;
            const GEntry en = s_ent[li * GWARPS + warp];
            if (!(en.code & 0xffffu)) continue;
            const TG* Gs = ringp + size_t(2 * slot + h) * A.sstride + (en.code >> 20) * GCOLS + 2 * lane;
            float2 W[GWN];
#pragma unroll
            for (int i = 0; i < GWN; i++) W[i] = Store<TG>::ld2(Gs + i * GCOLS);
            const float4* W4 = reinterpret_cast<const float4*>(s_wt + (size_t(k) * vcap + li) * GPL + q * GP);
            const float4 wa = W4[0], wb = W4[1];
            const uint32_t pid = (en.code >> 16) & 15u;
            if (pid < 8u) {  // fully visible planes
                switch (pid) {
                    case 0: g_taps4<0>(Z, W, wa, wb); break;
                    case 1: g_taps4<1>(Z, W, wa, wb); break;
                    case 2: g_taps4<2>(Z, W, wa, wb); break;
                    case 3: g_taps4<3>(Z, W, wa, wb); break;
                    case 4: g_taps4<4>(Z, W, wa, wb); break;
                    case 5: g_taps4<5>(Z, W, wa, wb); break;
                    default: g_taps4<6>(Z, W, wa, wb); break;
                }
            } else if (pid != uint32_t(kPatGen)) {
                // edge of the visible range: the adjoint zeroes the window
                // rows outside the view, the reference keeps per-plane rows
                if (ADJ) {
#pragma unroll
                    for (int i = 0; i < GWN; i++)
                        if (!((en.vm >> i) & 1u)) W[i] = make_float2(0.0f, 0.0f);
                }
                switch (pid) {
                    case 8: g_taps4_ivl<0>(Z, W, wa, wb, en.ivl); break;
                    case 9: g_taps4_ivl<1>(Z, W, wa, wb, en.ivl); break;
                    case 10: g_taps4_ivl<2>(Z, W, wa, wb, en.ivl); break;
                    case 11: g_taps4_ivl<3>(Z, W, wa, wb, en.ivl); break;
                    case 12: g_taps4_ivl<4>(Z, W, wa, wb, en.ivl); break;
                    case 13: g_taps4_ivl<5>(Z, W, wa, wb, en.ivl); break;
                    default: g_taps4_ivl<6>(Z, W, wa, wb, en.ivl); break;
                }
            } else {
                const float w0s[GP] = {wa.x, wa.z, wb.x, wb.z}, w1s[GP] = {wa.y, wa.w, wb.y, wb.w};
#pragma unroll
                for (int u = 0; u < GP; u++) {
                    const uint32_t c = (en.code >> (4 * u)) & 15u;
                    if (!(c & 3u)) continue;
                    const int o = int(c >> 2);
                    if ((c & 3u) == 1u) {
                        switch (o) {
                            case 0: g_taps<0, false>(Z[u], W, w0s[u], w1s[u], 0u, 0u); break;
                            case 1: g_taps<1, false>(Z[u], W, w0s[u], w1s[u], 0u, 0u); break;
                            default: g_taps<2, false>(Z[u], W, w0s[u], w1s[u], 0u, 0u); break;
                        }
                    } else {
                        // rows at the edge of the visible range: per-row masks
                        const uint32_t rows = (en.ivl >> (8 * u)) & 0xffu;
                        const uint32_t vm = ADJ ? en.vm : 0xffffffffu;
                        const uint32_t om = ADJ ? 0xffffffffu : rows;
                        switch (o) {
                            case 0: g_taps<0, true>(Z[u], W, w0s[u], w1s[u], vm, om); break;
                            case 1: g_taps<1, true>(Z[u], W, w0s[u], w1s[u], vm, om); break;
                            default: g_taps<2, true>(Z[u], W, w0s[u], w1s[u], vm, om); break;
                        }
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
        if (pr == nsp - 1) {
            if (!dead) store_view(k);
            pr = 0;
            k++;
        } else {
            pr++;
        }
    }
    // a tile that no slope reaches still writes its (zero) sums
    if (nsp == 0)
        for (int k = 0; k < nvw; k++) store_view(k);
    if (__syncthreads_or(dead)) {
        // a wait gave up: drain the copies still in flight
        if (tid == 0)
            for (int s = 0; s < ns; s++)
                if (s_round[s] >= 0) mbar_wait(&full[s], uint32_t(s_round[s] & 1), nullptr);
    }
}

struct XgatherArgs {
    petl_geom G;
    int step;        // view step of the members' view ranges
    int NUc;         // scratch row pitch
    int first;       // first chunk: the view sums start at zero, else at the partial sum
    int last;        // last chunk: write the volume, else the partial sum
    int accumulate;  // add to the volume instead of overwriting it
    float scale;
    Tables T;
    Members M;       // volumes (out) and views of the chunk
    int bplanes;     // planes of the scratch: numY, or 1 when its z sums do not depend on the plane
};

constexpr int XR = 4;         // volume rows z per k_bwd_xgather thread
constexpr int XMAXN = 1024;   // longest scratch / volume row

// x taps of a chunk of views into the volume: thread = column x of rows
// z0..z0+3 of plane y of one member, reading the two scratch taps of every
// view of that member straight from global memory (neighbouring threads
// share them through L1).  Grid (ceil(numX / 256), ceil(numZ / 4), numY x
// members).
template <int NM>
__global__ void __launch_bounds__(256) k_bwd_xgather(const float* __restrict__ B, float* __restrict__ part,
                                                     const XgatherArgs A)
{
    extern __shared__ Shift s_xs[];  // [views of the member] x shifts of plane y
    const petl_geom& G = A.G;
    const int NY = G.numY, NZ = G.numZ, NX = G.numX, NU0 = G.N_u0, NUc = A.NUc;
    const int mb = NM == 1 ? 0 : blockIdx.z / NY, y = blockIdx.z - mb * NY;
    const int x = blockIdx.x * 256 + threadIdx.x, z0 = blockIdx.y * XR;
    const int first = member_pick<NM>(A.M.first, mb), nvb = member_pick<NM>(A.M.nv, mb);
    float* __restrict__ f = static_cast<float*>(member_pick<NM>(A.M.out, mb));
    for (int vi = threadIdx.x; vi < nvb; vi += 256) s_xs[vi] = A.T.xt[size_t(first + vi * A.step) * NY + y];
    __syncthreads();
    if (x >= NX) return;
    const int nz = min(XR, NZ - z0);
    float acc[XR];
#pragma unroll
    for (int r = 0; r < XR; r++)
        acc[r] = (!A.first && r < nz) ? part[(size_t(z0 + r) * NY + y) * NX + x] : 0.0f;
    const int rlast = nz - 1;
    const int yb = A.bplanes == 1 ? 0 : y;  // the scratch plane of y
    const float* Bm = B + size_t(mb) * A.M.nvm * A.bplanes * NZ * NUc;
#pragma unroll 4
    for (int vi = 0; vi < nvb; vi++) {
        const Shift xs = s_xs[vi];
        const float wx1 = xs.w, wx0 = 1.0f - xs.w;
        const int j0 = x - xs.d;  // scratch column of tap 0
        const bool okm = unsigned(j0 - 1) < unsigned(NU0), ok0 = unsigned(j0) < unsigned(NU0);
        // in-bounds addresses for every tap; the out-of-range ones are selected away
        const int jm = min(max(j0 - 1, 0), NU0 - 1), jz = min(max(j0, 0), NU0 - 1);
        const float* Bv = Bm + ((size_t(vi) * A.bplanes + yb) * NZ + z0) * NUc;
#pragma unroll
        for (int r = 0; r < XR; r++) {
            const int rr = min(r, rlast);
            const float vm = __ldg(Bv + rr * NUc + jm), vz = __ldg(Bv + rr * NUc + jz);
            acc[r] = acc[r] + fmaf(wx1, okm ? vm : 0.0f, wx0 * (ok0 ? vz : 0.0f));
        }
    }
#pragma unroll
    for (int r = 0; r < XR; r++) {
        if (r >= nz) break;
        const size_t o = (size_t(z0 + r) * NY + y) * NX + x;
        if (!A.last)
            part[o] = acc[r];
        else
            f[o] = A.accumulate ? f[o] + A.scale * acc[r] : A.scale * acc[r];
    }
}

// z sums of one slope with v1 = 0 (the rebinned planogram of FBP), whose
// z taps and visible rows are the same on every plane: B[view][z][c] =
// S (1 - w) g[z - d][c] then + S w g[z - d - 1][c], the operations and
// masks of k_bwd_zgather for a single slope (rows outside the planogram
// read zero; the adjoint zeroes rows outside the visible u1 range and
// columns outside the view's visible u0 range, the reference semantics
// leave rows z outside the voxel test at zero).  Thread = column c of row z
// of one view; grid (ceil(N_u0 / 256), numZ, views).
struct FlatArgs {
    petl_geom G;
    int iv1;    // the slope
    int first;  // first view
    int step;   // view step
    int NUc;    // scratch row pitch
    Tables T;
};

template <bool ADJ>
__global__ void __launch_bounds__(256) k_bwd_zflat(const float* __restrict__ g, float* __restrict__ B, const FlatArgs A)
{
    const petl_geom& G = A.G;
    const int c = blockIdx.x * 256 + threadIdx.x, z = blockIdx.y, vi = blockIdx.z;
    if (c >= G.N_u0) return;
    const int v0 = A.first + vi * A.step;
    const Shift zs = A.T.zt[size_t(A.iv1) * G.numY];  // plane 0: every plane has the same
    const float S = A.T.S[size_t(A.iv1) * G.N_v0 + v0];
    const float w0 = S * (1.0f - zs.w), w1 = S * zs.w;
    const int2 ub1 = A.T.ub1[A.iv1];
    auto row = [&](int r) {
        const bool in = r >= 0 && r < G.N_u1 && (!ADJ || (r >= ub1.x && r <= ub1.y));
        return in ? g[((size_t(A.iv1) * G.N_v0 + v0) * G.N_u1 + r) * G.N_u0 + c] : 0.0f;
    };
    float zsum = 0.0f;
    bool live;
    if (ADJ) {
        live = true;
    } else {
        const int2 zv = A.T.zvis[size_t(A.iv1) * G.numY];
        live = z >= zv.x && z <= zv.y;
    }
    if (live) zsum = fmaf(w1, row(z - zs.d - 1), fmaf(w0, row(z - zs.d), 0.0f));
    if (ADJ) {
        const int2 u0r = A.T.ub0[v0];
        if (c < u0r.x || c > u0r.y) zsum = 0.0f;
    }
    B[(size_t(vi) * G.numZ + z) * A.NUc + c] = zsum;
}

int backproject_flat(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                     const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    const int n_v0 = vr.n_v0(G.N_v0);
    if (n_v0 <= 0 || n_v0 > 4096 || n_v0 > 65535 || G.N_u0 > XMAXN || G.numZ > 65535 || G.numY > 65535)
        return kNotApplicable;
    const int NUc = (G.N_u0 + 3) & ~3;
    float* B = nullptr;
    if (scratch_alloc(reinterpret_cast<void**>(&B), size_t(n_v0) * G.numZ * NUc * 4, st) != cudaSuccess) {
        cudaGetLastError();
        return kNotApplicable;
    }
    const FlatArgs FA{G, vr.iv1_begin, vr.iv0_first, vr.iv0_step, NUc, T};
    const dim3 grid(ceil_div(G.N_u0, 256), unsigned(G.numZ), unsigned(n_v0));
    if (mode == PETL_BP_ADJOINT)
        k_bwd_zflat<true><<<grid, 256, 0, st>>>(g, B, FA);
    else
        k_bwd_zflat<false><<<grid, 256, 0, st>>>(g, B, FA);
    note_launch();
    Members M;
    M.nb = 1;
    M.nvm = n_v0;
    M.first[0] = vr.iv0_first;
    M.nv[0] = n_v0;
    M.out[0] = f;
    const XgatherArgs X{G, vr.iv0_step, NUc, 1, 1, accumulate, scale, T, M, 1};
    k_bwd_xgather<1><<<dim3(ceil_div(G.numX, 256), ceil_div(G.numZ, XR), unsigned(G.numY)), 256,
                       size_t(n_v0) * sizeof(Shift), st>>>(B, nullptr, X);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(B, st);
    if (e != cudaSuccess) {
        set_error(std::string("backproject_flat: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace

// Backprojection of the members' views.  One member: its views in chunks of
// at most the scratch budget (and chunk_cap); several: one chunk, else
// kNotApplicable.  Member b reads planogram M0.in[b] and writes (or adds to)
// volume M0.out[b].
template <class TG>
int backproject_split_m(const petl_geom& G, const Members& M0, int mode, int accumulate, float scale,
                        const ViewRange& vr, const Tables& T, cudaStream_t st, int chunk_cap, const ChunkHook* hook)
{
    constexpr int EB = int(sizeof(TG));
    const int nb = M0.nb;
    if (nb < 1 || nb > kMaxMembers) return kNotApplicable;
    int nvmax = 0;
    for (int b = 0; b < nb; b++) nvmax = std::max(nvmax, M0.nv[b]);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (nvmax <= 0 || nv1 <= 0 || nv1 > GV1MAX) return kNotApplicable;
    // one slope at v1 = 0 (FBP's rebinned planogram): z sums without a plane
    // dimension
    if (std::is_same<TG, float>::value && nb == 1 && nv1 == 1 && M0.first[0] == vr.iv0_first &&
        M0.nv[0] == vr.n_v0(G.N_v0) && std::fmaf(float(vr.iv1_begin), G.T_v1, G.v1_0) == 0.0f)
        return backproject_flat(G, static_cast<const float*>(M0.in[0]), static_cast<float*>(M0.out[0]), mode,
                                accumulate, scale, vr, T, st);
    // the scratch holds a volume per view whatever the slope count: below
    // about ten slopes (the 2-D backprojection of FBP has one) the
    // single-pass kernel is cheaper than that round trip
    if (nv1 < kSplitMinSlopes) return kNotApplicable;
    // tensor map rows: a multiple of 16 bytes from a 16-byte aligned base
    if ((G.N_u0 * EB) % 16 != 0) return kNotApplicable;
    for (int b = 0; b < nb; b++)
        if ((reinterpret_cast<uintptr_t>(M0.in[b]) & 15) != 0) return kNotApplicable;
    if (G.N_u0 > XMAXN || G.numY > 65535 || G.numZ > 65535 * XR) return kNotApplicable;
    if (size_t(G.numY) * nb > 65535) return kNotApplicable;  // k_bwd_xgather grid.z
    const double step = double(std::max(std::fabs(G.v1_0), std::fabs(G.v1_0 + (G.N_v1 - 1) * G.T_v1))) *
                        double(G.T_x) / double(G.T_z);  // shift change per plane
    if (shift_spread(GP - 1, step) > GDW) return kNotApplicable;
    const int brb = GROWS + 1 + shift_spread(GPL - 1, step);
    if (brb > 254) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;

    ZgatherArgs A{};
    A.G = G;
    A.vr = vr;
    A.n_colblk = int(ceil_div(G.N_u0, GCOLS));
    A.n_rowblk = int(ceil_div(G.numZ, GROWS));
    A.brb = brb;
    A.sstride = (brb + 2) * GCOLS;  // a multiple of 64 elements: 128-byte aligned slopes
    A.NUc = (G.N_u0 + 3) & ~3;
    A.v1cap = nv1;
    A.T = T;
    A.err = err;
    A.wait_limit = wait_limit();

    // chunks of views whose scratch fits the budget, balanced in size
    const size_t per_view = size_t(G.numY) * G.numZ * A.NUc * 4;
    const size_t fit = std::max<size_t>(1, split_scratch_budget() / per_view);
    int nv, nchunks;
    if (nb == 1) {
        nv = int(std::min<size_t>(size_t(nvmax), fit));
        nv = std::min(nv, 4096);  // k_bwd_xgather stages the chunk's x shifts in shared memory
        if (chunk_cap > 0) nv = std::min(nv, chunk_cap);
        nchunks = (nvmax + nv - 1) / nv;
        nv = (nvmax + nchunks - 1) / nchunks;
    } else {
        if (size_t(nb) * nvmax > fit || nvmax > 4096 || chunk_cap > 0) return kNotApplicable;
        nv = nvmax;
        nchunks = 1;
    }
    A.vg = std::min(GVG, nv);
    if (size_t(ceil_div(nv, A.vg)) * nb > 65535) return kNotApplicable;  // grid.y

    const size_t fixed = size_t(nv1) * GWARPS * sizeof(GEntry) + size_t(A.vg) * nv1 * GPL * 8 + size_t(nv1) * 8 +
                         2 * GNSMAX * 8 + 8 + GNSMAX * 4;
    const size_t stage = size_t(2) * A.sstride * EB;
    A.ns = int(std::min<size_t>(GNSMAX, (227 * 1024 - std::min<size_t>(fixed, 227 * 1024)) / stage));
    if (A.ns < 2) return kNotApplicable;
    const size_t smem = size_t(A.ns) * stage + fixed;

    GMaps<kMaxMembers> maps;
    std::memset(&maps, 0, sizeof(maps));
    const uint64_t dims[4] = {uint64_t(G.N_u0), uint64_t(G.N_u1), uint64_t(G.N_v0), uint64_t(G.N_v1)};
    const uint64_t strides[3] = {uint64_t(G.N_u0) * EB, uint64_t(G.N_u0) * G.N_u1 * EB,
                                 uint64_t(G.N_u0) * G.N_u1 * G.N_v0 * EB};
    const uint32_t box[4] = {uint32_t(GCOLS), uint32_t(brb), 1u, 1u};
    for (int b = 0; b < nb; b++)
        if (!encode_tensor_map(&maps.m[b], M0.in[b], 4, dims, strides, box, EB)) return kNotApplicable;

    float* B = nullptr;
    float* part = nullptr;
    const size_t nvox = size_t(G.numX) * G.numY * G.numZ;
    if (scratch_alloc(reinterpret_cast<void**>(&B), per_view * nv * nb, st) != cudaSuccess ||
        (nchunks > 1 && scratch_alloc(reinterpret_cast<void**>(&part), nvox * 4, st) != cudaSuccess)) {
        cudaGetLastError();  // out of memory is not sticky: the caller takes the single-pass kernel
        if (B) cudaFreeAsync(B, st);
        return kNotApplicable;
    }
    const bool adj = mode == PETL_BP_ADJOINT;
    // kernels compiled for one member where there is one
    GMaps<1> map1;
    map1.m[0] = maps.m[0];
    auto kz1 = adj ? k_bwd_zgather<true, TG, 1> : k_bwd_zgather<false, TG, 1>;
    auto kzm = adj ? k_bwd_zgather<true, TG, kMaxMembers> : k_bwd_zgather<false, TG, kMaxMembers>;
    auto kx = nb == 1 ? k_bwd_xgather<1> : k_bwd_xgather<kMaxMembers>;
    cudaError_t e = nb == 1 ? cudaFuncSetAttribute(kz1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))
                            : cudaFuncSetAttribute(kzm, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    const unsigned ntile = unsigned(A.n_colblk) * unsigned(A.n_rowblk) * ceil_div(G.numY, GPL);
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
        if (hook && hook->fn) hook->fn(hook->ctx, vi0, nvc);
        A.M = M;
        A.gpm = int(ceil_div(nvc, A.vg));
        if (nb == 1)
            kz1<<<dim3(ntile, unsigned(A.gpm)), GNT, smem, st>>>(map1, B, A);
        else
            kzm<<<dim3(ntile, unsigned(A.gpm) * unsigned(nb)), GNT, smem, st>>>(maps, B, A);
        note_launch();
        XgatherArgs X{G, vr.iv0_step, A.NUc, c == 0, c == nchunks - 1, accumulate, scale, T, M, G.numY};
        kx<<<dim3(ceil_div(G.numX, 256), ceil_div(G.numZ, XR), unsigned(G.numY) * unsigned(nb)), 256,
                        size_t(nvc) * sizeof(Shift), st>>>(B, part, X);
        note_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(B, st);
    if (part) cudaFreeAsync(part, st);
    if (e != cudaSuccess) {
        set_error(std::string("backproject_split: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

template <class TG>
int backproject_split_t(const petl_geom& G, const TG* g, float* f, int mode, int accumulate, float scale,
                        const ViewRange& vr, const Tables& T, cudaStream_t st, int chunk_cap, const ChunkHook* hook)
{
    Members M;
    M.nb = 1;
    M.first[0] = vr.iv0_first;
    M.nv[0] = vr.n_v0(G.N_v0);
    M.in[0] = g;
    M.out[0] = f;
    return backproject_split_m<TG>(G, M, mode, accumulate, scale, vr, T, st, chunk_cap, hook);
}

int backproject_split(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                      const ViewRange& vr, const Tables& T, cudaStream_t st, int chunk_cap, const ChunkHook* hook)
{
    return backproject_split_t<float>(G, g, f, mode, accumulate, scale, vr, T, st, chunk_cap, hook);
}

int backproject_split_bf16(const petl_geom& G, const __nv_bfloat16* g, float* f, int mode, int accumulate,
                           float scale, const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    return backproject_split_t<__nv_bfloat16>(G, g, f, mode, accumulate, scale, vr, T, st, 0, nullptr);
}

int backproject_split_members(const petl_geom& G, const Members& M, int mode, int accumulate, float scale,
                              const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    return backproject_split_m<float>(G, M, mode, accumulate, scale, vr, T, st, 0, nullptr);
}

}  // namespace shear
}  // namespace petl
