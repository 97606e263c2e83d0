// Split forward projector for any psi (voxel height equal to the u1 bin
// pitch), the counterpart of the shear-warp split kernels
// (projector_split.cu) for orientations whose rays are not parallel to a
// volume axis.
//
// The reference footprint (src/projectors.cu:11-238) of a ray at its
// driving plane p (y = const for a y-driven view, x = const for an
// x-driven one, |r_x| < |r_y| deciding per view v0) is the product of a u0
// box overlap that depends on the ray parameter t and the in-plane voxel
// index a, and a u1 box overlap that depends on t, the slope v1 and the
// voxel row z.  t = (coordinate of plane p - p-coordinate of u0) / r_p
// depends on (v0, u0, p) only.  So
//   g[v1][v0][u1][u0] = l_phi rs sum_p sum_z w1(t, v1, u1, z) X[v0][p][z][u0],
//   X[v0][p][z][u0]   = sum_a w0(t, a, u0) f(z, p, a),
// and the two sums run as two kernels:
//
// * k_gx: a block stages 8 volume rows of plane p (from the volume, or from
//   its x/y-transposed copy for x-driven views) in shared memory; a thread
//   per column u0 evaluates the u0 taps of its ray on plane p once (the
//   reference's tap range and box overlaps, taps with a positive weight)
//   and applies them to the 8 rows.
// * k_gz: CTA = one view x 16 slopes x 64 rows x 32 columns, 16 warps of
//   2 slopes x 32 rows, one column per lane (a last block of at most 8
//   slopes as 8 slopes x 128 rows).  With equal pitch the u1 taps
//   of row u1 are voxel rows u1 + s and u1 + s + 1 with weights 1 - fr and
//   fr, where s + fr = (u1_0 - z_0 - t v1) / T_u1 depends on the lane's t
//   and the slope but not on the row.  The lanes' shifts differ, so each
//   lane reads its own rows of the staged plane: the rows every lane and
//   slope of the tile needs (bounded on the host) for 32 columns, row-major,
//   so a lane's column is its bank whatever its row.  They arrive per plane
//   by a tiled TMA copy (no multicast; rows outside the scratch read zero)
//   into a ring of three planes with full/empty mbarriers and a rotating
//   issuer; every wait is bounded (a wait that gives up sets the device
//   error word, the CTA drains its copies and writes nothing).
// Epilogue: scale l_phi * rs, the reference's ray masks, optional MLEM
// ratio.
//
// The sums are associated differently from the reference's (u0 taps summed
// before the z taps), so results agree with it to float rounding, not bit
// for bit.
#include <algorithm>
#include <cmath>
#include <string>

#include "common.cuh"
#include "gsplit.cuh"
#include "projector.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {

namespace {

constexpr int GXZ = 8;        // volume rows per k_gx block
constexpr int GZS = 16;       // slopes per k_gz CTA (2 per warp), main shape
constexpr int GZR = 64;       // rows per k_gz CTA (32 per warp), main shape
constexpr int GZS_T = 8;      // slopes per CTA of the tail shape (a last slope block of at most 8)
constexpr int GZR_T = 128;    // rows per CTA of the tail shape
constexpr int GZC = 32;       // columns per k_gz CTA (one per lane)
constexpr int GZT = 512;      // threads per k_gz CTA
constexpr int GJS = 2;        // slopes per warp
constexpr int GRW = 32;       // rows per warp (GZS / GJS x GZR / GRW = 16 warps; GZS_T / GJS x GZR_T / GRW the same;
                              // 16 rows per warp: 10 % slower at psi = 30, 256x256x128)
constexpr int GZRMAX = 224;   // staged rows per plane at most (TMA box rows <= 256)
constexpr int GZNS = 3;       // ring stages (one plane each) at most

struct GxArgs {
    petl_geom G;
    ViewRange vr;
    int vi0;    // first view of the chunk (index in vr)
    int NPmax;  // planes per view slot of the scratch
    int NUc;    // scratch row pitch
};

struct GzArgs {
    petl_geom G;
    ViewRange vr;
    int vi0;
    int NPmax;
    int NUc;
    int n_colblk, n_rowblk;
    int nrows;  // staged rows per plane (32 + shift range + margins, <= GZRMAX)
    int ns;     // ring stages
    int* err;
    unsigned wait_limit;  // bound of the waits on staged data (wait_limit(): kWaitLimit or 0)
};

__device__ __forceinline__ bool view_xdriven(const petl_geom& G, int iv0)
{
    return ray_geom(G, 0, iv0, 0, 0).xdriven;
}

// X[vi][p][z][u0] for 8 rows z of plane p of one view.  Grid (ceil(NZ / 8),
// NPmax, views of the chunk); dynamic shared memory 8 rows of the longest
// in-plane axis.
__global__ void __launch_bounds__(256) k_gx(const float* __restrict__ f, const float* __restrict__ fT,
                                           float* __restrict__ X, const GxArgs A)
{
    extern __shared__ float rowbuf[];
    const petl_geom& G = A.G;
    const int z0 = blockIdx.x * GXZ, p = blockIdx.y, vi = blockIdx.z;
    const int iv0 = A.vr.iv0_first + (A.vi0 + vi) * A.vr.iv0_step;
    const bool xd = view_xdriven(G, iv0);
    const int NP = xd ? G.numX : G.numY, NA = xd ? G.numY : G.numX;
    if (p >= NP) return;
    const float* __restrict__ src = xd ? fT : f;  // [z][p][a]
    const int nz = min(GXZ, G.numZ - z0);
    for (int e = threadIdx.x; e < nz * NA; e += blockDim.x) {
        const int r = e / NA, a = e - r * NA;
        rowbuf[r * NA + a] = src[(size_t(z0 + r) * NP + p) * NA + a];
    }
    __syncthreads();
    float* Xv = X + (size_t(vi) * A.NPmax + p) * G.numZ * A.NUc;
    for (int iu0 = threadIdx.x; iu0 < G.N_u0; iu0 += blockDim.x) {
        const RayGeom r = ray_geom(G, 0, iv0, 0, iu0);
        const PlaneTaps pt = xd ? plane_taps_x(G, r, p) : plane_taps_y(G, r, p);
        float acc[GXZ];
#pragma unroll
        for (int k = 0; k < GXZ; k++) acc[k] = 0.0f;
        for (int a = pt.a_min; a <= pt.a_max; a++) {
            const float w0 = xd ? tap_w0_x(G, r, pt.t, a, iu0) : tap_w0_y(G, r, pt.t, a, iu0);
            if (!(w0 > 0.0f)) continue;
#pragma unroll
            for (int k = 0; k < GXZ; k++) acc[k] = fmaf(w0, rowbuf[k * NA + a], acc[k]);
        }
        for (int k = 0; k < nz; k++) Xv[size_t(z0 + k) * A.NUc + iu0] = acc[k];
    }
}


// NQ slope pairs x (16 / NQ) row groups of 32 per CTA: NQ = 8 is the main
// shape (16 slopes x 64 rows), NQ = 4 the tail shape (8 slopes x 128 rows)
// for a last block of few slopes, which would leave most warps of a
// 16-slope CTA idle.
template <int NQ>
__global__ void __launch_bounds__(GZT, 1) k_gz(const __grid_constant__ CUtensorMap xmap, float* __restrict__ g,
                                                const float* __restrict__ meas, const GzArgs A)
{
    constexpr int SZ = NQ * GJS, RZ = (GZT / 32 / NQ) * GRW;
    extern __shared__ __align__(128) unsigned char gsm[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = warp % NQ, rg = warp / NQ;
    int t_ = blockIdx.x;
    const int colblk = t_ % A.n_colblk;
    t_ /= A.n_colblk;
    const int rowblk = t_ % A.n_rowblk;
    const int v1blk = t_ / A.n_rowblk;
    const int vi = blockIdx.y;
    const int iv0 = A.vr.iv0_first + (A.vi0 + vi) * A.vr.iv0_step;
    const int col0 = colblk * GZC, iu0 = col0 + lane;
    const int row0c = rowblk * RZ, row0 = row0c + rg * GRW;
    const int v1c = A.vr.iv1_begin + v1blk * SZ;           // first slope of the CTA
    const int v1c_last = min(v1c + SZ, A.vr.iv1_end) - 1;  // last slope of the CTA
    const int v1w = v1c + q * GJS;                          // first slope of the warp
    const int nrows = A.nrows, ns = A.ns;
    const float Tu1_inv = __frcp_rn(G.T_u1);
    const float K = fmul(fsub(G.u1_0, G.z_0), Tu1_inv);  // -(row 0 position) at t = 0
    // the lane's ray geometry on this view (t depends on v0, u0 and the plane)
    const RayGeom r = ray_geom(G, 0, iv0, 0, min(iu0, G.N_u0 - 1));
    const int NP = r.xdriven ? G.numX : G.numY;
    float v1s[GJS];
#pragma unroll
    for (int j = 0; j < GJS; j++) v1s[j] = fmul(ffma(float(min(v1w + j, A.vr.iv1_end - 1)), G.T_v1, G.v1_0), Tu1_inv);

    float* ring = reinterpret_cast<float*>(gsm);                        // [ns][nrows][32]
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + size_t(ns) * nrows * GZC);
    uint64_t* empty = full + GZNS;
    int* s_wr = reinterpret_cast<int*>(empty + GZNS);  // [GZNS] first staged row of the slot's plane
    int* s_round = s_wr + GZNS;                        // [GZNS] round of the copy last started in a slot
    volatile int* s_abort = s_round + GZNS;
    if (tid == 0) {
        for (int k = 0; k < ns; k++) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], GZT / 32);
            s_round[k] = -1;
        }
        *s_abort = 0;
        fence_barrier_init();
    }
    __syncthreads();

    // first staged row of plane p: the smallest shift at the tile's corners
    // (monotone in t and in v1), less one row of margin
    const float v1lo = fmul(ffma(float(v1c), G.T_v1, G.v1_0), Tu1_inv);
    const float v1hi = fmul(ffma(float(v1c_last), G.T_v1, G.v1_0), Tu1_inv);
    auto first_row = [&](int p) {
        const RayGeom ra = ray_geom(G, 0, iv0, 0, col0);
        const RayGeom rb = ray_geom(G, 0, iv0, 0, min(col0 + GZC - 1, G.N_u0 - 1));
        const float ta = plane_t(G, ra, p), tb = plane_t(G, rb, p);
        const float m = fminf(fminf(fmaf(-ta, v1lo, K), fmaf(-ta, v1hi, K)), fminf(fmaf(-tb, v1lo, K), fmaf(-tb, v1hi, K)));
        return row0c + int(floorf(m)) - 1;
    };
    const uint32_t box_bytes = uint32_t(nrows) * GZC * 4u;
    auto issue = [&](int p) {
        const int slot = p % ns, round = p / ns;
        if (round > 0 && !mbar_wait(&empty[slot], uint32_t((round - 1) & 1), A.err, A.wait_limit)) return false;
        if (*s_abort) return false;
        fence_proxy_async_smem();
        const int wr = first_row(p);
        s_wr[slot] = wr;
        mbar_arrive_expect_tx(&full[slot], box_bytes);
        tma_load_3d(ring + size_t(slot) * nrows * GZC, &xmap, &full[slot], col0, wr, vi * A.NPmax + p);
        s_round[slot] = round;
        return true;
    };
    if (tid == 0)
        for (int p = 0; p < ns - 1 && p < NP; p++) issue(p);
    // the next plane this warp starts: the first p >= ns - 1 with p % 16 == warp
    constexpr int NW = GZT / 32;
    int my_next = warp + NW * ((ns - 1 - warp + NW - 1) / NW);
    if (my_next < ns - 1) my_next += NW;

    float acc[GJS][GRW];
#pragma unroll
    for (int j = 0; j < GJS; j++)
#pragma unroll
        for (int k = 0; k < GRW; k++) acc[j][k] = 0.0f;

    bool dead = false;
    int slot = 0;
    uint32_t phase = 0;
    for (int p = 0; p < NP; p++) {
        if (p + ns - 1 == my_next) {
            if (lane == 0 && !dead && my_next < NP && !issue(my_next)) dead = true;
            my_next += NW;
        }
        if (!dead) dead = !mbar_wait(&full[slot], phase, A.err, A.wait_limit);
        if (dead) *s_abort = 1;  // before this warp releases the slot
        if (!dead) {
            const float tt = plane_t(G, r, p);
            const float* B = ring + size_t(slot) * nrows * GZC + lane;
            const int wr = s_wr[slot];
#pragma unroll
            for (int j = 0; j < GJS; j++) {
                const float nc = fmaf(-tt, v1s[j], K);
                const float sf = floorf(nc);
                const float fr = nc - sf, w0 = 1.0f - fr;
                int base = row0 + int(sf) - wr;  // staged row of tap 0 of the warp's first row
                if (base < 0 || base + GRW + 1 > nrows) {  // outside the staged rows: the host bound failed
                    atomicOr(A.err, kErrLayout);
                    base = 0;
                }
                float W[GRW + 1];
#pragma unroll
                for (int k = 0; k < GRW + 1; k++) W[k] = B[(base + k) * GZC];
#pragma unroll
                for (int k = 0; k < GRW; k++) acc[j][k] = fmaf(fr, W[k + 1], fmaf(w0, W[k], acc[j][k]));
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
            for (int k = 0; k < ns; k++)
                if (s_round[k] >= 0) mbar_wait(&full[k], uint32_t(s_round[k] & 1), nullptr);
        return;
    }

    // epilogue: scale, ray masks, optional MLEM ratio
    if (iu0 >= G.N_u0) return;
#pragma unroll
    for (int j = 0; j < GJS; j++) {
        const int iv1 = v1w + j;
        if (iv1 >= A.vr.iv1_end) continue;
#pragma unroll
        for (int k = 0; k < GRW; k++) {
            const int iu1 = row0 + k;
            if (iu1 >= G.N_u1) continue;
            const RayGeom rr = ray_geom(G, iv1, iv0, iu1, iu0);
            const float val = ray_visible(G, iv1, iv0, iu1, iu0) ? fmul(fmul(acc[j][k], rr.l_phi), rr.rs) : 0.0f;
            const size_t o = ((size_t(iv1) * G.N_v0 + iv0) * G.N_u1 + iu1) * G.N_u0 + iu0;
            g[o] = meas ? ratio_rule(__ldg(&meas[o]), val) : val;
        }
    }
}

}  // namespace


__global__ void k_transpose_xy(const float* __restrict__ in, float* __restrict__ out, int nx, int ny)
{
    __shared__ float tile[32][33];
    const int z = blockIdx.z, x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const float* fz = in + size_t(z) * nx * ny;
    float* tz = out + size_t(z) * nx * ny;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int y = y0 + j, x = x0 + threadIdx.x;
        if (y < ny && x < nx) tile[j][threadIdx.x] = fz[size_t(y) * nx + x];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int x = x0 + j, y = y0 + threadIdx.x;
        if (x < nx && y < ny) tz[size_t(x) * ny + y] = tile[threadIdx.x][j];
    }
}

// kNotApplicable when the layout rules fail (the caller then runs the
// general kernel): voxel height != u1 pitch, a view whose shift range over a
// tile exceeds the staged rows, or scratch that cannot be allocated.
int project_gsplit(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                   cudaStream_t st)
{
    constexpr int kNotApplicable = -2;
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return 0;
    if (G.T_z != G.T_u1 || G.N_u0 > 4096 || G.numX > 4096 || G.numY > 4096) return kNotApplicable;
    // staged rows per plane: the CTA's rows + the range of floor(-c0) over a
    // tile's 32 columns and its slopes + margins.  -c0 = (u1_0 - z_0 + t v1)
    // / T_u1 with t = (coordinate of the plane - u0 pscale) * inv: bounded
    // with the extremes of |t| and of its change over 32 columns.
    const double vmax = std::max(std::fabs(double(G.v1_0)), std::fabs(double(G.v1_0) + (G.N_v1 - 1) * double(G.T_v1)));
    const double xext = std::max(std::fabs(double(G.x_0)), std::fabs(double(G.x_0) + (G.numX - 1) * double(G.T_x)));
    const double yext = std::max(std::fabs(double(G.y_0)), std::fabs(double(G.y_0) + (G.numY - 1) * double(G.T_x)));
    const double uext = std::max(std::fabs(double(G.u0_0)), std::fabs(double(G.u0_0) + (G.N_u0 - 1) * double(G.T_u0)));
    double tmax = 0, dtmax = 0;
    bool any_xd = false;
    for (int k = 0; k < n_v0; k++) {
        const HostView h = host_view(G, vr.iv0_first + k * vr.iv0_step);
        any_xd = any_xd || h.xd;
        tmax = std::max(tmax, (std::max(xext, yext) + uext * h.pscale) * std::fabs(h.inv));
        dtmax = std::max(dtmax, GZC * double(G.T_u0) * h.pscale * std::fabs(h.inv));
    }
    auto staged_rows = [&](int slopes, int rows) {
        const double dv1 = (slopes - 1) * std::fabs(double(G.T_v1));
        const double spread = (dtmax * vmax + tmax * dv1 + dtmax * dv1) / double(G.T_u1);
        return rows + int(std::ceil(spread * (1.0 + 1e-6))) + 5;  // + floors and the one-row margins
    };
    const int nrows = staged_rows(GZS, GZR);
    if (nrows > GZRMAX) return kNotApplicable;
    // a last block of at most 8 slopes runs in the tail shape
    const int rem = nv1 % GZS;
    const int nrows_t = staged_rows(GZS_T, GZR_T);
    const bool tail = rem > 0 && rem <= GZS_T && nrows_t <= GZRMAX && G.N_u1 > GZR;
    const int nv1_main = tail ? nv1 - rem : nv1;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;

    const int NPmax = any_xd ? std::max(G.numX, G.numY) : G.numY;
    const int NUc = (G.N_u0 + 3) & ~3;
    const size_t per_view = size_t(NPmax) * G.numZ * NUc * 4;
    int nv = int(std::max<size_t>(1, std::min<size_t>(size_t(n_v0), gsplit_scratch_budget() / per_view)));
    nv = std::min(nv, 65535);
    const int nchunks = (n_v0 + nv - 1) / nv;
    nv = (n_v0 + nchunks - 1) / nchunks;
    float* X = nullptr;
    float* fT = nullptr;
    if (scratch_alloc(reinterpret_cast<void**>(&X), per_view * nv, st) != cudaSuccess ||
        (any_xd && scratch_alloc(reinterpret_cast<void**>(&fT), size_t(G.numX) * G.numY * G.numZ * 4, st) !=
                       cudaSuccess)) {
        cudaGetLastError();
        if (X) cudaFreeAsync(X, st);
        return kNotApplicable;
    }
    cudaError_t e = cudaSuccess;
    if (any_xd) {
        k_transpose_xy<<<dim3(ceil_div(G.numX, 32), ceil_div(G.numY, 32), unsigned(G.numZ)), dim3(32, 8), 0, st>>>(
            f, fT, G.numX, G.numY);
        note_launch();
    }
    const int NAmax = any_xd ? std::max(G.numX, G.numY) : G.numX;
    const size_t xsmem = size_t(GXZ) * NAmax * 4;
    e = cudaFuncSetAttribute(k_gx, cudaFuncAttributeMaxDynamicSharedMemorySize, int(xsmem));
    // one z launch shape: its argument block, tensor map (boxes of 32
    // columns x its staged rows; TMA, no multicast; rows outside read zero)
    // and shared memory
    struct ZLaunch {
        GzArgs Z;
        CUtensorMap map;
        size_t smem;
        unsigned nblk;
    };
    auto z_setup = [&](ZLaunch& L, int rows_cta, int slopes_cta, int staged, int v1b, int v1e) -> cudaError_t {
        const size_t stage = size_t(staged) * GZC * 4;
        const int ns = int(std::min<size_t>(GZNS, (200 * 1024) / stage));
        if (ns < 2) return cudaErrorInvalidValue;
        L.smem = size_t(ns) * stage + GZNS * 16 + GZNS * 8 + 16;
        L.Z = GzArgs{};
        L.Z.G = G;
        L.Z.vr = vr;
        L.Z.vr.iv1_begin = v1b;
        L.Z.vr.iv1_end = v1e;
        L.Z.NPmax = NPmax;
        L.Z.NUc = NUc;
        L.Z.n_colblk = int(ceil_div(G.N_u0, GZC));
        L.Z.n_rowblk = int(ceil_div(G.N_u1, rows_cta));
        L.Z.nrows = staged;
        L.Z.ns = ns;
        L.Z.err = err;
        L.Z.wait_limit = wait_limit();
        L.nblk = unsigned(L.Z.n_colblk) * unsigned(L.Z.n_rowblk) * ceil_div(v1e - v1b, slopes_cta);
        const uint64_t dims[3] = {uint64_t(NUc), uint64_t(G.numZ), uint64_t(NPmax) * uint64_t(nv)};
        const uint64_t strides[2] = {uint64_t(NUc) * 4, uint64_t(NUc) * G.numZ * 4};
        const uint32_t box[3] = {uint32_t(GZC), uint32_t(staged), 1u};
        return encode_tensor_map(&L.map, X, 3, dims, strides, box, 4) ? cudaSuccess : cudaErrorInvalidValue;
    };
    ZLaunch zm{}, zt{};
    if (e == cudaSuccess && nv1_main > 0) e = z_setup(zm, GZR, GZS, nrows, vr.iv1_begin, vr.iv1_begin + nv1_main);
    if (e == cudaSuccess && tail) e = z_setup(zt, GZR_T, GZS_T, nrows_t, vr.iv1_begin + nv1_main, vr.iv1_end);
    if (e == cudaSuccess && nv1_main > 0)
        e = cudaFuncSetAttribute(k_gz<GZS / GJS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(zm.smem));
    if (e == cudaSuccess && tail)
        e = cudaFuncSetAttribute(k_gz<GZS_T / GJS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(zt.smem));
    for (int c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int vi0 = c * nv, nvc = std::min(nv, n_v0 - vi0);
        const GxArgs XA{G, vr, vi0, NPmax, NUc};
        k_gx<<<dim3(ceil_div(G.numZ, GXZ), unsigned(NPmax), unsigned(nvc)), 256, xsmem, st>>>(f, fT, X, XA);
        note_launch();
        if (nv1_main > 0) {
            zm.Z.vi0 = vi0;
            k_gz<GZS / GJS><<<dim3(zm.nblk, unsigned(nvc)), GZT, zm.smem, st>>>(zm.map, g, meas, zm.Z);
            note_launch();
        }
        if (tail) {
            zt.Z.vi0 = vi0;
            k_gz<GZS_T / GJS><<<dim3(zt.nblk, unsigned(nvc)), GZT, zt.smem, st>>>(zt.map, g, meas, zt.Z);
            note_launch();
        }
        e = cudaGetLastError();
    }
    cudaFreeAsync(X, st);
    if (fT) cudaFreeAsync(fT, st);
    if (e != cudaSuccess) {
        set_error(std::string("project_gsplit: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl
