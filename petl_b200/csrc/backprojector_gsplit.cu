// Split exact-adjoint backprojector for any psi (voxel height equal to the
// u1 bin pitch): the transpose of the split forward projector
// (projector_gsplit.cu), whose footprint factors as
//   g[v1][v0][u1][u0] = l_phi rs vis sum_p sum_z w1(t, v1, u1, z) X[v0][p][z][u0],
//   X[v0][p][z][u0]   = sum_a w0(t, a, u0) f(z, p, a),
// with t = t(v0, u0, p) and, at equal pitch, w1 the pair (1 - fr, fr) on
// rows u1 + s, u1 + s + 1 (s + fr = (u1_0 - z_0 - t v1) / T_u1).  Its
// transpose runs as
//   h[v0][v1][u1][u0] = g l_phi rs vis                         (k_gprep)
//   Y[v0][p][z][u0]   = sum_v1 fr h[z - s - 1] + (1 - fr) h[z - s]  (k_gzT)
//   f(z, p, a)       += sum_v0 sum_u0 w0(t, a, u0) Y[v0][p][z][u0]  (k_gxT)
// with the forward's own shift, weights and tap functions, so that the pair
// is the exact transpose up to float rounding (the general adjoint kernel,
// k_backproject_adj_general, enumerates the same taps per voxel).
//
// * k_gzT mirrors k_gz with the roles of slopes and planes swapped: CTA = one
//   view x 16 planes x 64 voxel rows x 32 columns, 16 warps of 2 planes x 32
//   rows, one column per lane; the loop runs over the slopes, whose rows of
//   h (the rows every lane and plane of the tile needs, bounded on the host)
//   arrive by tiled TMA copies (no multicast; rows outside the planogram read
//   zero) into a ring of three slopes with full/empty mbarriers, a rotating
//   issuer and bounded waits (a wait that gives up sets the device error
//   word, the CTA drains its copies and writes nothing).
// * k_gxT: block = one driving plane x 16 voxel rows x 256 in-plane voxels;
//   per view it stages the rows of Y over the u0 columns that reach its
//   voxels and a table of each column's u0 taps (first voxel, up to four
//   weights, computed by plane_taps and tap_w0 as the forward does); a
//   thread per voxel sums the columns whose taps include it in ascending u0,
//   the views in ascending order (deterministic, no atomics).  y-driven
//   views accumulate into f's layout, x-driven ones into an x/y-transposed
//   volume; k_gcombine adds both into f with the scale.
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

constexpr int TZP = 16;      // planes per k_gzT CTA (2 per warp)
constexpr int TZR = 64;      // voxel rows per k_gzT CTA (32 per warp)
constexpr int TZC = 32;      // columns per k_gzT CTA (one per lane)
constexpr int TZT = 512;     // threads per k_gzT CTA
constexpr int TJP = 2;       // planes per warp
constexpr int TRW = 32;      // rows per warp (TZP / TJP x TZR / TRW = 16 warps; 16 rows: 21 % slower at psi = 30)
constexpr int TZRMAX = 224;  // staged rows per slope at most (TMA box rows <= 256)
constexpr int TZNS = 3;      // ring stages (one slope each) at most
constexpr int TXA = 256;     // in-plane voxels per k_gxT block (one per thread)
constexpr int TXZ = 16;      // voxel rows per k_gxT block
constexpr int TMAXT = 4;     // u0 taps of one column on one plane at most

struct GprepArgs {
    petl_geom G;
    ViewRange vr;
    int vi0, nvc;  // chunk: first view (index in vr), views
    int NUc;
};

struct GzTArgs {
    petl_geom G;
    ViewRange vr;
    int vi0;
    int NPmax, NUc;
    int n_colblk, n_rowblk;
    int nrows;  // staged rows per slope (32 + shift range + margins, <= TZRMAX)
    int ns;     // ring stages
    int* err;
    unsigned wait_limit;
};

struct GxTArgs {
    petl_geom G;
    ViewRange vr;
    int vi0, nvc;
    int NPmax, NUc;
    int want_xd;  // 1: x-driven views into the transposed volume; 0: y-driven views into f's layout
    int UW;       // staged u0 columns per view at most
    int add;      // 1: add to the output (a later chunk of views)
    int* err;
};

// h[vi][v1 - v1_begin][u1][c] = g l_phi rs on visible rays, 0 elsewhere
// (columns N_u0 .. NUc - 1 included).  l_phi and rs depend on the view and
// the slope only; grid (column blocks, (view, slope) slabs), both strided.
__global__ void k_gprep(const float* __restrict__ g, float* __restrict__ h, const GprepArgs A)
{
    const petl_geom& G = A.G;
    const int nv1 = A.vr.iv1_end - A.vr.iv1_begin;
    const int per = G.N_u1 * A.NUc;  // elements per slab
    for (int slab = blockIdx.y; slab < A.nvc * nv1; slab += gridDim.y) {
        const int vi = slab / nv1, jv1 = slab - vi * nv1;
        const int iv1 = A.vr.iv1_begin + jv1;
        const int iv0 = A.vr.iv0_first + (A.vi0 + vi) * A.vr.iv0_step;
        const RayGeom rr = ray_geom(G, iv1, iv0, 0, 0);
        const float* gs = g + (size_t(iv1) * G.N_v0 + iv0) * G.N_u1 * G.N_u0;
        float* hs = h + size_t(slab) * per;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < per; e += gridDim.x * blockDim.x) {
            const int iu1 = e / A.NUc, c = e - iu1 * A.NUc;
            float val = 0.0f;
            if (c < G.N_u0 && ray_visible(G, iv1, iv0, iu1, c))
                val = fmul(fmul(__ldg(&gs[size_t(iu1) * G.N_u0 + c]), rr.l_phi), rr.rs);
            hs[e] = val;
        }
    }
}

__global__ void __launch_bounds__(TZT, 1) k_gzT(const __grid_constant__ CUtensorMap hmap, float* __restrict__ Y,
                                                 const GzTArgs A)
{
    extern __shared__ __align__(128) unsigned char tsm[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = warp % (TZP / TJP), rg = warp / (TZP / TJP);
    int t_ = blockIdx.x;
    const int colblk = t_ % A.n_colblk;
    t_ /= A.n_colblk;
    const int rowblk = t_ % A.n_rowblk;
    const int pblk = t_ / A.n_rowblk;
    const int vi = blockIdx.y;
    const int iv0 = A.vr.iv0_first + (A.vi0 + vi) * A.vr.iv0_step;
    const int col0 = colblk * TZC, iu0 = col0 + lane;
    const int row0c = rowblk * TZR, row0 = row0c + rg * TRW;
    // the lane's ray geometry on this view (t depends on v0, u0 and the plane)
    const RayGeom r = ray_geom(G, 0, iv0, 0, min(iu0, G.N_u0 - 1));
    const int NP = r.xdriven ? G.numX : G.numY;
    const int p0c = pblk * TZP;
    if (p0c >= NP) return;  // the whole CTA: its planes lie beyond this view's driving axis
    const int p_last = min(p0c + TZP, NP) - 1;
    const int pw = p0c + q * TJP;  // first plane of the warp
    const int nv1 = A.vr.iv1_end - A.vr.iv1_begin;
    const int nrows = A.nrows, ns = A.ns;
    const float Tu1_inv = __frcp_rn(G.T_u1);
    const float K = fmul(fsub(G.u1_0, G.z_0), Tu1_inv);  // -(row 0 position) at t = 0
    float ts[TJP];
#pragma unroll
    for (int j = 0; j < TJP; j++) ts[j] = plane_t(G, r, min(pw + j, NP - 1));

    float* ring = reinterpret_cast<float*>(tsm);  // [ns][nrows][32]
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + size_t(ns) * nrows * TZC);
    uint64_t* empty = full + TZNS;
    int* s_wr = reinterpret_cast<int*>(empty + TZNS);  // [TZNS] first staged row of the slot's slope
    int* s_round = s_wr + TZNS;                        // [TZNS] round of the copy last started in a slot
    volatile int* s_abort = s_round + TZNS;
    if (tid == 0) {
        for (int k = 0; k < ns; k++) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], TZT / 32);
            s_round[k] = -1;
        }
        *s_abort = 0;
        fence_barrier_init();
    }
    __syncthreads();

    // corner ray parameters of the tile (t is monotone in the plane and in u0)
    const RayGeom ra = ray_geom(G, 0, iv0, 0, col0);
    const RayGeom rb = ray_geom(G, 0, iv0, 0, min(col0 + TZC - 1, G.N_u0 - 1));
    const float tc[4] = {plane_t(G, ra, p0c), plane_t(G, ra, p_last), plane_t(G, rb, p0c), plane_t(G, rb, p_last)};
    // first staged row of slope jv1: row0c - 1 - (the largest shift over the
    // tile's corners), less one row of margin
    auto first_row = [&](int jv1) {
        const float v1s = fmul(ffma(float(A.vr.iv1_begin + jv1), G.T_v1, G.v1_0), Tu1_inv);
        float m = fmaf(-tc[0], v1s, K);
#pragma unroll
        for (int k = 1; k < 4; k++) m = fmaxf(m, fmaf(-tc[k], v1s, K));
        return row0c - int(floorf(m)) - 2;
    };
    const uint32_t box_bytes = uint32_t(nrows) * TZC * 4u;
    auto issue = [&](int jv1) {
        const int slot = jv1 % ns, round = jv1 / ns;
        if (round > 0 && !mbar_wait(&empty[slot], uint32_t((round - 1) & 1), A.err, A.wait_limit)) return false;
        if (*s_abort) return false;
        fence_proxy_async_smem();
        const int wr = first_row(jv1);
        s_wr[slot] = wr;
        mbar_arrive_expect_tx(&full[slot], box_bytes);
        tma_load_3d(ring + size_t(slot) * nrows * TZC, &hmap, &full[slot], col0, wr, vi * nv1 + jv1);
        s_round[slot] = round;
        return true;
    };
    if (tid == 0)
        for (int jv1 = 0; jv1 < ns - 1 && jv1 < nv1; jv1++) issue(jv1);
    // the next slope this warp starts: the first jv1 >= ns - 1 with jv1 % 16 == warp
    constexpr int NW = TZT / 32;
    int my_next = warp + NW * ((ns - 1 - warp + NW - 1) / NW);
    if (my_next < ns - 1) my_next += NW;

    float acc[TJP][TRW];
#pragma unroll
    for (int j = 0; j < TJP; j++)
#pragma unroll
        for (int k = 0; k < TRW; k++) acc[j][k] = 0.0f;

    bool dead = false, layout_bad = false;
    int slot = 0;
    uint32_t phase = 0;
    for (int jv1 = 0; jv1 < nv1; jv1++) {
        if (jv1 + ns - 1 == my_next) {
            if (lane == 0 && !dead && my_next < nv1 && !issue(my_next)) dead = true;
            my_next += NW;
        }
        if (!dead) dead = !mbar_wait(&full[slot], phase, A.err, A.wait_limit);
        if (dead) *s_abort = 1;  // before this warp releases the slot
        if (!dead) {
            const float v1s = fmul(ffma(float(A.vr.iv1_begin + jv1), G.T_v1, G.v1_0), Tu1_inv);
            const float* B = ring + size_t(slot) * nrows * TZC + lane;
            const int wr = s_wr[slot];
#pragma unroll
            for (int j = 0; j < TJP; j++) {
                // the forward's shift and weights for (plane, slope, column)
                const float nc = fmaf(-ts[j], v1s, K);
                const float sf = floorf(nc);
                const float fr = nc - sf, w0 = 1.0f - fr;
                int base = row0 - int(sf) - 1 - wr;  // staged row of h[z - s - 1] for the warp's first row z
                // outside the staged rows (the host bound failed): read row 0,
                // report once after the loop
                const bool bad = base < 0 || base + TRW + 1 > nrows;
                layout_bad |= bad;
                base = bad ? 0 : base;
                float W[TRW + 1];
#pragma unroll
                for (int k = 0; k < TRW + 1; k++) W[k] = B[(base + k) * TZC];
#pragma unroll
                for (int k = 0; k < TRW; k++) acc[j][k] = fmaf(w0, W[k + 1], fmaf(fr, W[k], acc[j][k]));
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
        if (++slot == ns) {
            slot = 0;
            phase ^= 1u;
        }
    }
    if (layout_bad) atomicOr(A.err, kErrLayout);
    if (__syncthreads_or(dead)) {
        // a wait gave up: drain the copies still in flight, write nothing
        if (tid == 0)
            for (int k = 0; k < ns; k++)
                if (s_round[k] >= 0) mbar_wait(&full[k], uint32_t(s_round[k] & 1), nullptr);
        return;
    }

    if (iu0 >= G.N_u0) return;
#pragma unroll
    for (int j = 0; j < TJP; j++) {
        const int p = pw + j;
        if (p >= NP) continue;
        float* Yp = Y + (size_t(vi) * A.NPmax + p) * G.numZ * A.NUc + iu0;
#pragma unroll
        for (int k = 0; k < TRW; k++) {
            const int z = row0 + k;
            if (z < G.numZ) Yp[size_t(z) * A.NUc] = acc[j][k];
        }
    }
}

// out[z][p][a] (+)= sum over the chunk's views of the class want_xd of
// sum_u0 w0(t, a, u0) Y[vi][p][z][u0].  Grid (ceil(NA / 256) x
// ceil(numZ / 16), NP); 256 threads; dynamic shared memory
// UW x (16 + 4 + 1) words.
__global__ void __launch_bounds__(TXA) k_gxT(const float* __restrict__ Y, float* __restrict__ out, const GxTArgs A)
{
    extern __shared__ float xsm[];
    const petl_geom& G = A.G;
    const int UW = A.UW;
    float* Ys = xsm;                                      // [TXZ][UW]
    float* Wt = Ys + TXZ * UW;                            // [TMAXT][UW]
    int* amin = reinterpret_cast<int*>(Wt + TMAXT * UW);  // [UW]
    const bool xd = A.want_xd != 0;
    const int NP = xd ? G.numX : G.numY, NA = xd ? G.numY : G.numX;
    const int nach = (NA + TXA - 1) / TXA;
    const int ach = blockIdx.x % nach, zb = blockIdx.x / nach;
    const int p = blockIdx.y;
    const int tid = threadIdx.x;
    const int a0 = ach * TXA, a = a0 + tid, alast = min(a0 + TXA, NA) - 1;
    const int z0 = zb * TXZ, nz = min(TXZ, G.numZ - z0);
    const float pc = ffma(float(p), G.T_x, xd ? G.x_0 : G.y_0);  // coordinate of the driving plane
    const float Tu0_inv = __frcp_rn(G.T_u0);
    float acc[TXZ];
#pragma unroll
    for (int k = 0; k < TXZ; k++) acc[k] = 0.0f;

    for (int vi = 0; vi < A.nvc; vi++) {
        const int iv0 = A.vr.iv0_first + (A.vi0 + vi) * A.vr.iv0_step;
        const RayGeom r0 = ray_geom(G, 0, iv0, 0, 0);
        if (r0.xdriven != xd) continue;  // uniform over the block
        // u0 bin (continuous index) of the ray through the centre of voxel aa
        // of this plane: u0 = x r_y - y r_x.  A column iu0 has a positive tap
        // on the voxel only if |iu0 - c| < (fw + 1/2) |r_p trig|, r_p the
        // driving component and trig the cos (y-driven) or sin (x-driven)
        // that scales the tap; h adds half a bin of margin for rounding.
        auto cpos = [&](int aa) {
            const float ac = ffma(float(aa), G.T_x, xd ? G.y_0 : G.x_0);
            const float x = xd ? pc : ac, y = xd ? ac : pc;
            return fmul(fsub(fsub(fmul(x, r0.ry), fmul(y, r0.rx)), G.u0_0), Tu0_inv);
        };
        const float stretch = xd ? fabsf(fmul(r0.rx, G.sin_psi)) : fabsf(fmul(r0.ry, G.cos_psi));
        const float h = ffma(fadd(r0.fw, 0.5f), stretch, 0.5f);
        const float c_lo = cpos(a0), c_hi = cpos(alast);
        const int ulo = max(0, int(floorf(fsub(fminf(c_lo, c_hi), h))));
        int uhi = min(G.N_u0 - 1, int(ceilf(fadd(fmaxf(c_lo, c_hi), h))));
        if (uhi < ulo) continue;  // uniform: no column of this view reaches the block
        if (uhi - ulo + 1 > UW) {  // the host bound failed
            if (tid == 0) atomicOr(A.err, kErrLayout);
            uhi = ulo + UW - 1;
        }
        const int nu = uhi - ulo + 1;
        __syncthreads();  // the previous view's reads are done
        const float* Yv = Y + ((size_t(vi) * A.NPmax + p) * G.numZ + z0) * A.NUc + ulo;
        for (int e = tid; e < nz * nu; e += TXA) {
            const int k = e / nu, u = e - k * nu;
            Ys[k * UW + u] = Yv[size_t(k) * A.NUc + u];
        }
        for (int u = tid; u < nu; u += TXA) {
            const int iu0 = ulo + u;
            const RayGeom r = ray_geom(G, 0, iv0, 0, iu0);
            const PlaneTaps pt = xd ? plane_taps_x(G, r, p) : plane_taps_y(G, r, p);
            if (pt.a_max - pt.a_min + 1 > TMAXT) atomicOr(A.err, kErrLayout);  // the host bound failed
            amin[u] = pt.a_min;
#pragma unroll
            for (int j = 0; j < TMAXT; j++) {
                const int aa = pt.a_min + j;
                float w = 0.0f;
                if (aa <= pt.a_max) {
                    w = xd ? tap_w0_x(G, r, pt.t, aa, iu0) : tap_w0_y(G, r, pt.t, aa, iu0);
                    if (!(w > 0.0f)) w = 0.0f;
                }
                Wt[j * UW + u] = w;
            }
        }
        __syncthreads();
        if (a < NA) {
            const float c = cpos(a);
            const int j0 = max(ulo, int(floorf(fsub(c, h)))), j1 = min(uhi, int(ceilf(fadd(c, h))));
            for (int iu = j0; iu <= j1; iu++) {
                const int u = iu - ulo, j = a - amin[u];
                if (unsigned(j) >= unsigned(TMAXT)) continue;
                const float w = Wt[j * UW + u];
                if (!(w > 0.0f)) continue;
#pragma unroll
                for (int k = 0; k < TXZ; k++) acc[k] = fmaf(w, Ys[k * UW + u], acc[k]);
            }
        }
    }
    if (a >= NA) return;
#pragma unroll
    for (int k = 0; k < TXZ; k++) {
        if (k >= nz) break;
        const size_t o = (size_t(z0 + k) * NP + p) * NA + a;
        out[o] = A.add ? fadd(out[o], acc[k]) : acc[k];
    }
}

// f[z][y][x] = (accumulate ? f : 0) + scale (S[z][y][x] + ST[z][x][y]); S or
// ST null when no view of its class ran.  Grid (ceil(nx / 32), ceil(ny / 32),
// nz); block (32, 8).
__global__ void k_gcombine(float* __restrict__ f, const float* __restrict__ S, const float* __restrict__ ST,
                           int accumulate, float scale, int nx, int ny)
{
    __shared__ float tile[32][33];
    const int z = blockIdx.z, x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const size_t slice = size_t(z) * nx * ny;
    if (ST) {
        for (int j = threadIdx.y; j < 32; j += blockDim.y) {
            const int x = x0 + j, y = y0 + threadIdx.x;
            if (x < nx && y < ny) tile[j][threadIdx.x] = ST[slice + size_t(x) * ny + y];
        }
        __syncthreads();
    }
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int y = y0 + j, x = x0 + threadIdx.x;
        if (y >= ny || x >= nx) continue;
        const size_t o = slice + size_t(y) * nx + x;
        float v = S ? S[o] : 0.0f;
        if (ST) v = fadd(v, tile[threadIdx.x][j]);
        const float r = fmul(v, scale);
        f[o] = accumulate ? fadd(f[o], r) : r;
    }
}

}  // namespace

// kNotApplicable when the layout rules fail (the caller then runs the
// general adjoint kernel): voxel height != u1 pitch, u0 pitch above twice
// the voxel width (more than four taps per column), a tile whose shift range
// exceeds the staged rows, or scratch that cannot be allocated.
int backproject_gsplit_adjoint(const petl_geom& G, const float* g, float* f, int accumulate, float scale,
                               const ViewRange& vr, cudaStream_t st)
{
    constexpr int kNotApplicable = -2;
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return kNotApplicable;
    if (G.T_z != G.T_u1 || G.N_u0 > 4096 || G.numX > 4096 || G.numY > 4096) return kNotApplicable;
    // a column's tap range on a plane spans (T_u0 |trig| + T_x) / T_x voxels:
    // at most TMAXT taps when T_u0 <= 2 T_x (one voxel of margin for rounding)
    if (double(G.T_u0) / double(G.T_x) + 2.01 > TMAXT) return kNotApplicable;
    // staged rows per slope: 32 + the range of floor(nc) over a tile's 16
    // planes and 32 columns + margins; nc = K - t v1 / T_u1 with t
    // changing by T_x |inv| per plane and T_u0 pscale |inv| per column
    const double vmax = std::max(std::fabs(double(G.v1_0)), std::fabs(double(G.v1_0) + (G.N_v1 - 1) * double(G.T_v1)));
    double spread = 0, uw = 0;
    bool any_xd = false, any_yd = false;
    for (int k = 0; k < n_v0; k++) {
        const HostView hv = host_view(G, vr.iv0_first + k * vr.iv0_step);
        (hv.xd ? any_xd : any_yd) = true;
        const double ainv = std::fabs(hv.inv);
        const double dt = ((TZP - 1) * double(G.T_x) + (TZC - 1) * double(G.T_u0) * hv.pscale) * ainv;
        spread = std::max(spread, dt * vmax / double(G.T_u1));
        // u0 columns reaching a block's 256 voxels of one plane
        const double trig = std::fabs(double(hv.xd ? G.sin_psi : G.cos_psi));
        const double fw = 0.5 * double(G.T_x) / (trig * double(G.T_u0));
        const double h = (fw + 0.5) * trig / ainv + 0.5;
        uw = std::max(uw, (TXA - 1) * double(G.T_x) / (double(G.T_u0) * ainv) + 2 * h + 4);
    }
    const int nrows = TZR + int(std::ceil(spread * (1.0 + 1e-6))) + 5;  // + floors and the one-row margins
    if (nrows > TZRMAX) return kNotApplicable;
    const int UW = (int(std::ceil(uw * (1.0 + 1e-6))) + 31) & ~31;
    const size_t xsmem = size_t(UW) * (TXZ + TMAXT + 1) * 4;
    if (xsmem > 160 * 1024) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;

    const int NPmax = any_xd ? std::max(G.numX, G.numY) : G.numY;
    const int NUc = (G.N_u0 + 3) & ~3;
    const size_t per_view = (size_t(NPmax) * G.numZ + size_t(nv1) * G.N_u1) * NUc * 4;
    int nv = int(std::max<size_t>(1, std::min<size_t>(size_t(n_v0), gsplit_scratch_budget() / per_view)));
    nv = std::min(nv, 65535);
    if (size_t(nv) * nv1 > (size_t(1) << 31)) nv = std::max(1, int((size_t(1) << 31) / nv1));
    const int nchunks = (n_v0 + nv - 1) / nv;
    nv = (n_v0 + nchunks - 1) / nchunks;
    const size_t nvox = size_t(G.numX) * G.numY * G.numZ;
    float* Y = nullptr;
    float* H = nullptr;
    float* S = nullptr;
    float* ST = nullptr;
    if (scratch_alloc(reinterpret_cast<void**>(&Y), size_t(NPmax) * G.numZ * NUc * 4 * nv, st) != cudaSuccess ||
        scratch_alloc(reinterpret_cast<void**>(&H), size_t(nv1) * G.N_u1 * NUc * 4 * nv, st) != cudaSuccess ||
        (any_yd && scratch_alloc(reinterpret_cast<void**>(&S), nvox * 4, st) != cudaSuccess) ||
        (any_xd && scratch_alloc(reinterpret_cast<void**>(&ST), nvox * 4, st) != cudaSuccess)) {
        cudaGetLastError();
        for (float* q : {Y, H, S, ST})
            if (q) cudaFreeAsync(q, st);
        return kNotApplicable;
    }
    cudaError_t e = cudaFuncSetAttribute(k_gxT, cudaFuncAttributeMaxDynamicSharedMemorySize, int(xsmem));
    const size_t stage = size_t(nrows) * TZC * 4;
    const int ns = int(std::min<size_t>(TZNS, (200 * 1024) / stage));
    const size_t zsmem = size_t(ns) * stage + TZNS * 16 + TZNS * 8 + 16;
    if (ns < 2) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gzT, cudaFuncAttributeMaxDynamicSharedMemorySize, int(zsmem));
    GzTArgs Z{};
    Z.G = G;
    Z.vr = vr;
    Z.NPmax = NPmax;
    Z.NUc = NUc;
    Z.n_colblk = int(ceil_div(G.N_u0, TZC));
    Z.n_rowblk = int(ceil_div(G.numZ, TZR));
    Z.nrows = nrows;
    Z.ns = ns;
    Z.err = err;
    Z.wait_limit = wait_limit();
    // h as a 3-D tensor: columns, u1 rows, view slot x slope; boxes of 32
    // columns x nrows rows (TMA, no multicast; rows outside read zero)
    CUtensorMap map;
    const uint64_t dims[3] = {uint64_t(NUc), uint64_t(G.N_u1), uint64_t(nv1) * uint64_t(nv)};
    const uint64_t strides[2] = {uint64_t(NUc) * 4, uint64_t(NUc) * G.N_u1 * 4};
    const uint32_t box[3] = {uint32_t(TZC), uint32_t(nrows), 1u};
    if (e == cudaSuccess && !encode_tensor_map(&map, H, 3, dims, strides, box, 4)) e = cudaErrorInvalidValue;
    const unsigned zblk = unsigned(Z.n_colblk) * unsigned(Z.n_rowblk) * ceil_div(NPmax, TZP);
    for (int c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int vi0 = c * nv, nvc = std::min(nv, n_v0 - vi0);
        const GprepArgs P{G, vr, vi0, nvc, NUc};
        const unsigned gx = unsigned(std::min<size_t>(ceil_div(size_t(G.N_u1) * NUc, size_t(256)), 32));
        const unsigned gy = unsigned(std::min<size_t>(size_t(nvc) * nv1, 8192));
        k_gprep<<<dim3(gx, gy), 256, 0, st>>>(g, H, P);
        note_launch();
        Z.vi0 = vi0;
        k_gzT<<<dim3(zblk, unsigned(nvc)), TZT, zsmem, st>>>(map, Y, Z);
        note_launch();
        for (int cls = 0; cls < 2; cls++) {
            const bool xd = cls == 1;
            if (!(xd ? any_xd : any_yd)) continue;
            const int NP = xd ? G.numX : G.numY, NA = xd ? G.numY : G.numX;
            const GxTArgs XA{G, vr, vi0, nvc, NPmax, NUc, int(xd), UW, int(c > 0), err};
            k_gxT<<<dim3(unsigned(ceil_div(NA, TXA) * ceil_div(G.numZ, TXZ)), unsigned(NP)), TXA, xsmem, st>>>(
                Y, xd ? ST : S, XA);
            note_launch();
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_gcombine<<<dim3(ceil_div(G.numX, 32), ceil_div(G.numY, 32), unsigned(G.numZ)), dim3(32, 8), 0, st>>>(
            f, S, ST, accumulate, scale, G.numX, G.numY);
        note_launch();
        e = cudaGetLastError();
    }
    for (float* q : {Y, H, S, ST})
        if (q) cudaFreeAsync(q, st);
    if (e != cudaSuccess) {
        set_error(std::string("backproject_gsplit_adjoint: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl
