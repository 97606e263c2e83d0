// Separable-footprint projector and backprojectors for any planogram
// orientation and any voxel/bin pitch.
//
// These kernels restate the reference arithmetic (src/projectors.cu:11-377)
// without texture hardware: volume and planogram are read from global memory
// (both are L2-friendly in their access order), the backprojector's 2x2
// texture taps become exact bilinear weights, and all v1 slices run in one
// launch instead of one launch per slice.  The specialised shear kernels in
// projector_shear.cu take over the axis-aligned, equal-pitch case that the
// benchmarks use; these kernels serve every other geometry and the tests.
//
// Thread layout: the fastest thread index walks the fastest array index
// (u0 for planograms, x for volumes) so loads and stores coalesce.
#include "common.cuh"
#include "projector.cuh"

namespace petl {

// ---------------------------------------------------------------------------
// forward projection, one thread per ray
// ---------------------------------------------------------------------------
template <bool COUNT>
__global__ void __launch_bounds__(128)
k_project_general(const float* __restrict__ f, float* __restrict__ g, const petl_geom G, const ViewRange vr,
                  int n_v0, unsigned long long* __restrict__ nnz, const float* __restrict__ meas)
{
    const int iu0 = blockIdx.x * 32 + threadIdx.x;
    const int iu1 = blockIdx.y * 4 + threadIdx.y;
    const int view = blockIdx.z;
    const int iv1 = vr.iv1_begin + view / n_v0;
    const int iv0 = vr.iv0_first + (view % n_v0) * vr.iv0_step;
    const bool inside = iu0 < G.N_u0 && iu1 < G.N_u1;
    float val = 0.0f;
    unsigned long long cnt = 0;
    if (inside && ray_visible(G, iv1, iv0, iu1, iu0)) {
        const RayGeom rg = ray_geom(G, iv1, iv0, iu1, iu0);
        const int Nx = G.numX, Ny = G.numY;
        if (rg.xdriven) {
            for (int ix = 0; ix < Nx; ix++) {
                const PlaneTaps pt = plane_taps_x(G, rg, ix);
                for (int iy = pt.a_min; iy <= pt.a_max; iy++) {
                    const float w0 = tap_w0_x(G, rg, pt.t, iy, iu0);
                    if (w0 > 0.0f) {
                        for (int iz = pt.z_min; iz <= pt.z_max; iz++) {
                            const float w1 = tap_w1(G, rg, pt.t, iz, iu1);
                            if (w1 > 0.0f) {
                                if (COUNT) cnt++;
                                else val = ffma(__ldg(&f[(size_t(iz) * Ny + iy) * Nx + ix]), fmul(w0, w1), val);
                            }
                        }
                    }
                }
            }
        } else {
            for (int iy = 0; iy < Ny; iy++) {
                const PlaneTaps pt = plane_taps_y(G, rg, iy);
                for (int ix = pt.a_min; ix <= pt.a_max; ix++) {
                    const float w0 = tap_w0_y(G, rg, pt.t, ix, iu0);
                    if (w0 > 0.0f) {
                        for (int iz = pt.z_min; iz <= pt.z_max; iz++) {
                            const float w1 = tap_w1(G, rg, pt.t, iz, iu1);
                            if (w1 > 0.0f) {
                                if (COUNT) cnt++;
                                else val = ffma(__ldg(&f[(size_t(iz) * Ny + iy) * Nx + ix]), fmul(w0, w1), val);
                            }
                        }
                    }
                }
            }
        }
        val = fmul(fmul(val, rg.l_phi), rg.rs);
    }
    if (COUNT) {
        // warp-level reduction then one atomic per warp (counting only)
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nnz, cnt);
        return;
    }
    if (inside) {
        const size_t o = ((size_t(iv1) * G.N_v0 + iv0) * G.N_u1 + iu1) * G.N_u0 + iu0;
        g[o] = meas ? ratio_rule(__ldg(&meas[o]), val) : val;
    }
}

// ---------------------------------------------------------------------------
// reference-semantics backprojection, KZ voxels (z .. z+KZ-1) per thread: the
// voxels of a column share, per view, the u0 footprint (A, B), its range and
// l_phi, and their u1 rows overlap, so every planogram row of the column's
// union is summed over u0 once and combined per voxel with its own u1
// weights, in the order (ascending u1) and with the float operations of
// k_backproject_ref_general.  Columns whose union spans more than kRows
// rows take the per-voxel form.
// ---------------------------------------------------------------------------
// seven CTAs per SM (at most 73 registers, a few spilled) measured 25 %
// faster than four (128 registers): the kernel waits on its L1-resident
// gathers and needs the warps
template <int KZ>
__global__ void __launch_bounds__(128, 7)
k_backproject_ref_general_multi(const float* __restrict__ g, float* __restrict__ f, const petl_geom G,
                                const ViewRange vr, int accumulate, float scale)
{
    constexpr int kRows = 6;  // 4 voxels of equal pitch span at most 6 rows (8 measured 10 % slower)
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 4 + threadIdx.y;
    const int iz0 = blockIdx.z * KZ;
    if (ix >= G.numX || iy >= G.numY) return;
    const float cs = G.cos_psi, sn = G.sin_psi;
    const float x = fmaf(float(ix), G.T_x, G.x_0);
    const float y = fmaf(float(iy), G.T_x, G.y_0);
    float z[KZ];
#pragma unroll
    for (int k = 0; k < KZ; k++) z[k] = fmaf(float(iz0 + k), G.T_z, G.z_0);
    const float t = fmaf(y, cs, -(x * sn));
    const float x_dot_theta = fmaf(x, cs, y * sn);
    const float Tu1_inv = 1.0f / G.T_u1, Tu0_inv = 1.0f / G.T_u0;
    const float xdt_dy = 0.5f * G.T_x * sn, t_dy = 0.5f * G.T_x * cs;
    const float xdt_dx = 0.5f * G.T_x * cs, t_dx = -0.5f * G.T_x * sn;
    const size_t slab = size_t(G.N_v0) * G.N_u1 * G.N_u0;
    float acc[KZ];
#pragma unroll
    for (int k = 0; k < KZ; k++) acc[k] = 0.0f;
    for (int iv1 = vr.iv1_begin; iv1 < vr.iv1_end; iv1++) {
        const float v1 = fmaf(float(iv1), G.T_v1, G.v1_0);
        bool vis[KZ];
        float iu1_A[KZ], iu1_B[KZ];
        int ua[KZ], ub[KZ];
        int lo = 1 << 30, hi = -(1 << 30);
        bool anyv = false;
#pragma unroll
        for (int k = 0; k < KZ; k++) {
            const float u1 = fmaf(v1, t, z[k]);
            vis[k] = iz0 + k < G.numZ && (fabsf(u1) - 0.5f * G.T_u1 <= fmaf(-G.R, fabsf(v1), G.H));
            const float iu1_mid = (u1 - G.u1_0) * Tu1_inv;
            iu1_A[k] = iu1_mid - 0.5f * G.T_z * Tu1_inv;
            iu1_B[k] = iu1_mid + 0.5f * G.T_z * Tu1_inv;
            ua[k] = max(int(ceilf(iu1_A[k] - 0.5f)), 0);
            ub[k] = min(int(floorf(iu1_B[k] + 0.5f)), G.N_u1 - 1);
            if (vis[k] && ua[k] <= ub[k]) {
                lo = min(lo, ua[k]);
                hi = max(hi, ub[k]);
            }
            anyv = anyv || vis[k];
        }
        if (!anyv) continue;
        const float* gs = g + size_t(iv1) * slab;
        float val[KZ];
#pragma unroll
        for (int k = 0; k < KZ; k++) val[k] = 0.0f;
        if (hi - lo + 1 <= kRows) {
            // u1 weight of union row r for voxel k (0 outside its rows)
            float w1r[KZ][kRows];
#pragma unroll
            for (int k = 0; k < KZ; k++)
#pragma unroll
                for (int r = 0; r < kRows; r++) {
                    const int iu1 = lo + r;
                    w1r[k][r] = (vis[k] && iu1 >= ua[k] && iu1 <= ub[k])
                                    ? fmaxf(0.0f, fminf(float(iu1) + 0.5f, iu1_B[k]) - fmaxf(float(iu1) - 0.5f, iu1_A[k]))
                                    : 0.0f;
                }
            for (int iv0 = vr.iv0_first; iv0 < G.N_v0; iv0 += vr.iv0_step) {
                const float v0 = fmaf(float(iv0), G.T_v0, G.v0_0);
                const float wy = fmaf(v0, cs, sn);
                const float wx = fmaf(-v0, sn, cs);
                const float l_phi = 1.0f / fmaxf(fabsf(wy), fabsf(wx)) * rsqrtf(1.0f + v0 * v0 + v1 * v1);
                float A, B;
                if (fabsf(wy) > fabsf(wx)) {
                    const float lo_ = (x_dot_theta - xdt_dy + v0 * (t - t_dy) - G.u0_0) * Tu0_inv;
                    const float hi_ = (x_dot_theta + xdt_dy + v0 * (t + t_dy) - G.u0_0) * Tu0_inv;
                    A = wy >= 0.0f ? lo_ : hi_;
                    B = wy >= 0.0f ? hi_ : lo_;
                } else {
                    const float lo_ = (x_dot_theta - xdt_dx + v0 * (t - t_dx) - G.u0_0) * Tu0_inv;
                    const float hi_ = (x_dot_theta + xdt_dx + v0 * (t + t_dx) - G.u0_0) * Tu0_inv;
                    A = wx >= 0.0f ? lo_ : hi_;
                    B = wx >= 0.0f ? hi_ : lo_;
                }
                const int iu0_min = max(int(ceilf(A - 0.5f)), 0);
                const int iu0_max = min(int(floorf(B + 0.5f)), G.N_u0 - 1);
                const float* gv = gs + size_t(iv0) * G.N_u1 * G.N_u0;
                // the u0 weights do not depend on the row: evaluated once for
                // footprints of up to 4 bins (the same values in the same order)
                const int nw = iu0_max - iu0_min + 1;
                float w0a[4];
#pragma unroll
                for (int i = 0; i < 4; i++)
                    w0a[i] = fmaxf(0.0f, fminf(float(iu0_min + i) + 0.5f, B) - fmaxf(float(iu0_min + i) - 0.5f, A));
                float s0[kRows];
#pragma unroll
                for (int r = 0; r < kRows; r++) {
                    s0[r] = 0.0f;
                    if (lo + r > hi) continue;
                    const float* gr = gv + size_t(lo + r) * G.N_u0;
                    if (nw <= 4) {
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            if (i < nw) s0[r] = fmaf(w0a[i], __ldg(&gr[iu0_min + i]), s0[r]);
                    } else {
                        for (int iu0 = iu0_min; iu0 <= iu0_max; iu0++) {
                            const float w0 = fmaxf(0.0f, fminf(float(iu0) + 0.5f, B) - fmaxf(float(iu0) - 0.5f, A));
                            s0[r] = fmaf(w0, __ldg(&gr[iu0]), s0[r]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < KZ; k++) {
                    float sv = 0.0f;
#pragma unroll
                    for (int r = 0; r < kRows; r++)
                        if (w1r[k][r] > 0.0f) sv = fmaf(w1r[k][r], s0[r], sv);
                    val[k] = fmaf(sv, l_phi, val[k]);
                }
            }
        } else {
            for (int iv0 = vr.iv0_first; iv0 < G.N_v0; iv0 += vr.iv0_step) {
                const float v0 = fmaf(float(iv0), G.T_v0, G.v0_0);
                const float wy = fmaf(v0, cs, sn);
                const float wx = fmaf(-v0, sn, cs);
                const float l_phi = 1.0f / fmaxf(fabsf(wy), fabsf(wx)) * rsqrtf(1.0f + v0 * v0 + v1 * v1);
                float A, B;
                if (fabsf(wy) > fabsf(wx)) {
                    const float lo_ = (x_dot_theta - xdt_dy + v0 * (t - t_dy) - G.u0_0) * Tu0_inv;
                    const float hi_ = (x_dot_theta + xdt_dy + v0 * (t + t_dy) - G.u0_0) * Tu0_inv;
                    A = wy >= 0.0f ? lo_ : hi_;
                    B = wy >= 0.0f ? hi_ : lo_;
                } else {
                    const float lo_ = (x_dot_theta - xdt_dx + v0 * (t - t_dx) - G.u0_0) * Tu0_inv;
                    const float hi_ = (x_dot_theta + xdt_dx + v0 * (t + t_dx) - G.u0_0) * Tu0_inv;
                    A = wx >= 0.0f ? lo_ : hi_;
                    B = wx >= 0.0f ? hi_ : lo_;
                }
                const int iu0_min = max(int(ceilf(A - 0.5f)), 0);
                const int iu0_max = min(int(floorf(B + 0.5f)), G.N_u0 - 1);
                const float* gv = gs + size_t(iv0) * G.N_u1 * G.N_u0;
#pragma unroll
                for (int k = 0; k < KZ; k++) {
                    if (!vis[k]) continue;
                    float sv = 0.0f;
                    for (int iu1 = ua[k]; iu1 <= ub[k]; iu1++) {
                        const float w1 = fmaxf(0.0f, fminf(float(iu1) + 0.5f, iu1_B[k]) - fmaxf(float(iu1) - 0.5f, iu1_A[k]));
                        if (!(w1 > 0.0f)) continue;
                        float s0 = 0.0f;
                        for (int iu0 = iu0_min; iu0 <= iu0_max; iu0++) {
                            const float w0 = fmaxf(0.0f, fminf(float(iu0) + 0.5f, B) - fmaxf(float(iu0) - 0.5f, A));
                            s0 = fmaf(w0, __ldg(&gv[size_t(iu1) * G.N_u0 + iu0]), s0);
                        }
                        sv = fmaf(w1, s0, sv);
                    }
                    val[k] = fmaf(sv, l_phi, val[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < KZ; k++)
            if (vis[k]) acc[k] = fmaf(val[k], G.T_x, acc[k]);
    }
#pragma unroll
    for (int k = 0; k < KZ; k++) {
        if (iz0 + k >= G.numZ) break;
        const size_t o = (size_t(iz0 + k) * G.numY + iy) * G.numX + ix;
        const float r = acc[k] * scale;
        f[o] = accumulate ? f[o] + r : r;
    }
}

// ---------------------------------------------------------------------------
// exact adjoint of k_project_general, one thread per voxel (gather).
// For every view the candidate rays around the voxel's projection are
// enumerated and the forward projector's own tap test and weights are
// evaluated for them (same device functions, bit-identical weights).
// ---------------------------------------------------------------------------
// six CTAs per SM: 14 % faster than four at psi = 30
__global__ void __launch_bounds__(128, 6)
k_backproject_adj_general(const float* __restrict__ g, float* __restrict__ f, const petl_geom G, const ViewRange vr,
                          int accumulate, float scale)
{
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 4 + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= G.numX || iy >= G.numY) return;
    const double xd = double(G.x_0) + double(ix) * G.T_x;
    const double yd = double(G.y_0) + double(iy) * G.T_x;
    const double zd = double(G.z_0) + double(iz) * G.T_z;
    const double cs = G.cos_psi, sn = G.sin_psi;
    float acc = 0.0f;
    for (int iv1 = vr.iv1_begin; iv1 < vr.iv1_end; iv1++) {
        const size_t slab = size_t(iv1) * G.N_v0;
        for (int iv0 = vr.iv0_first; iv0 < G.N_v0; iv0 += vr.iv0_step) {
            const float v1f = ffma(float(iv1), G.T_v1, G.v1_0);
            const float v0f = ffma(float(iv0), G.T_v0, G.v0_0);
            // approximate continuous ray coordinates through the voxel centre
            const double v0 = v0f, v1 = v1f;
            const double rx = -(v0 * cs + sn), ry = -(v0 * sn - cs);
            const bool xdr = fabs(rx) >= fabs(ry);
            // solve p + t r = voxel for (u0, t) in the x-y plane, then u1
            // p = (u0 cs, u0 sn), r = (rx, ry): u0 = (x ry - y rx) / (cs ry - sn rx)
            // (cs*ry - sn*rx == 1 for this parametrisation)
            const double u0c = xd * ry - yd * rx;
            const double tc = xdr ? (xd - u0c * cs) / rx : (yd - u0c * sn) / ry;
            const double u1c = zd + v1 * tc;
            const double c0 = (u0c - G.u0_0) / G.T_u0, c1 = (u1c - G.u1_0) / G.T_u1;
            const double s0 = 0.5 * (xdr ? G.T_x / fabs(sn) : G.T_x / fabs(cs)) / G.T_u0 + 0.5 * G.T_u0 / G.T_u0;
            const int j0 = max(0, int(floor(c0 - s0 - 2.0))), j1 = min(G.N_u0 - 1, int(ceil(c0 + s0 + 2.0)));
            const double s1 = 0.5 * G.T_z / G.T_u1 + 0.5;
            const int k0 = max(0, int(floor(c1 - s1 - 2.0))), k1 = min(G.N_u1 - 1, int(ceil(c1 + s1 + 2.0)));
            float sview = 0.0f;
            for (int iu0 = j0; iu0 <= j1; iu0++) {
                for (int iu1 = k0; iu1 <= k1; iu1++) {
                    if (!ray_visible(G, iv1, iv0, iu1, iu0)) continue;
                    // the forward projector's own tap test for this ray
                    const RayGeom rg = ray_geom(G, iv1, iv0, iu1, iu0);
                    float w0;
                    PlaneTaps pt;
                    if (rg.xdriven) {
                        pt = plane_taps_x(G, rg, ix);
                        if (iy < pt.a_min || iy > pt.a_max) continue;
                        w0 = tap_w0_x(G, rg, pt.t, iy, iu0);
                    } else {
                        pt = plane_taps_y(G, rg, iy);
                        if (ix < pt.a_min || ix > pt.a_max) continue;
                        w0 = tap_w0_y(G, rg, pt.t, ix, iu0);
                    }
                    if (!(w0 > 0.0f) || iz < pt.z_min || iz > pt.z_max) continue;
                    const float w1 = tap_w1(G, rg, pt.t, iz, iu1);
                    if (!(w1 > 0.0f)) continue;
                    const float gy = __ldg(&g[((slab + iv0) * G.N_u1 + iu1) * G.N_u0 + iu0]);
                    sview = ffma(fmul(fmul(gy, fmul(w0, w1)), rg.l_phi), rg.rs, sview);
                }
            }
            acc = fadd(acc, sview);
        }
    }
    const size_t o = (size_t(iz) * G.numY + iy) * G.numX + ix;
    const float r = acc * scale;
    f[o] = accumulate ? f[o] + r : r;
}

int launch_project_general(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                           cudaStream_t st)
{
    const int n_v0 = vr.n_v0(G.N_v0);
    const long long nviews = (long long)(vr.iv1_end - vr.iv1_begin) * n_v0;
    if (nviews <= 0) return 0;
    PETL_REQUIRE(nviews <= 65535, "view count exceeds grid limit");
    dim3 block(32, 4, 1);
    dim3 grid(ceil_div(G.N_u0, 32), ceil_div(G.N_u1, 4), unsigned(nviews));
    k_project_general<false><<<grid, block, 0, st>>>(f, g, G, vr, n_v0, nullptr, meas);
    PETL_LAUNCH_CHECK("project_general");
    return 0;
}

int launch_count_nnz(const petl_geom& G, unsigned long long* d_count, cudaStream_t st)
{
    const long long nviews = (long long)G.N_v1 * G.N_v0;
    PETL_REQUIRE(nviews <= 65535, "view count exceeds grid limit");
    dim3 block(32, 4, 1);
    dim3 grid(ceil_div(G.N_u0, 32), ceil_div(G.N_u1, 4), unsigned(nviews));
    k_project_general<true><<<grid, block, 0, st>>>(nullptr, nullptr, G, ViewRange{0, G.N_v1, 0, 1}, G.N_v0, d_count,
                                                   nullptr);
    PETL_LAUNCH_CHECK("count_nnz");
    return 0;
}

int launch_backproject_general(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                               const ViewRange& vr, cudaStream_t st)
{
    PETL_REQUIRE(G.numZ <= 65535, "numZ exceeds grid limit");
    dim3 block(32, 4, 1);
    dim3 grid(ceil_div(G.numX, 32), ceil_div(G.numY, 4), unsigned(G.numZ));
    constexpr int KZ = 4;
    if (mode == PETL_BP_ADJOINT) {
        k_backproject_adj_general<<<grid, block, 0, st>>>(g, f, G, vr, accumulate, scale);
    } else {
        grid.z = ceil_div(G.numZ, KZ);
        k_backproject_ref_general_multi<KZ><<<grid, block, 0, st>>>(g, f, G, vr, accumulate, scale);
    }
    PETL_LAUNCH_CHECK("backproject_general");
    return 0;
}

}  // namespace petl
