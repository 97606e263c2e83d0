// Device-side pieces of the separable-footprint projector shared by the
// forward kernels and the exact-adjoint backprojector.
//
// The functions restate src/projectors.cu:11-238 of the reference: ray masks
// (lines 30-43), ray parametrisation p + t r (52-53), the per-plane tap range
// (95-101 / 150-156) and the box-overlap footprint weights (110-119 /
// 165-174).  Two deliberate differences: the in-plane coordinate of a tap is
// formed directly from its index instead of by running addition, and every
// weight is evaluated with rounding-pinned intrinsics, so the forward
// projector and its gather-form adjoint compute bit-identical weights.
#pragma once
#include "common.cuh"

namespace petl {

// The ray masks of the reference's forward kernel, evaluated in float with
// fused multiply-adds as the reference's compiled kernel evaluates them:
// the u0 test depends on (iv0, iu0) only, the u1 test on (iv1, iu1) only.
// Each holds on an interval of its bin index (the tests are monotone in
// |u0| and |u1|).
__device__ __forceinline__ bool u0_visible(const petl_geom& G, int iv0, int iu0)
{
    const float v0 = ffma(float(iv0), G.T_v0, G.v0_0);
    const float u0 = ffma(float(iu0), G.T_u0, G.u0_0);
    return !(fsub(fabsf(u0), fmul(0.5f, G.T_u0)) > ffma(G.R, fabsf(v0), G.L));
}

__device__ __forceinline__ bool u1_visible(const petl_geom& G, int iv1, int iu1)
{
    const float v1 = ffma(float(iv1), G.T_v1, G.v1_0);
    const float u1 = ffma(float(iu1), G.T_u1, G.u1_0);
    return !(fsub(fabsf(u1), fmul(0.5f, G.T_u1)) > ffma(-G.R, fabsf(v1), G.H));
}

__device__ __forceinline__ bool ray_visible(const petl_geom& G, int iv1, int iv0, int iu1, int iu0)
{
    return u0_visible(G, iv0, iu0) && u1_visible(G, iv1, iu1);
}

struct RayGeom {
    float px, py, pz, rx, ry, rz;
    float inv;       // 1/r.y (y-driven) or 1/r.x (x-driven)
    float trig_inv;  // 1/cos(psi) (y-driven) or 1/sin(psi) (x-driven)
    float width;     // half bin width projected on the driving plane
    float fw;        // half voxel width in u0 bin units
    float l_phi, rs;
    bool xdriven;
};

__device__ __forceinline__ RayGeom ray_geom(const petl_geom& G, int iv1, int iv0, int iu1, int iu0)
{
    RayGeom r;
    const float v1 = ffma(float(iv1), G.T_v1, G.v1_0);
    const float v0 = ffma(float(iv0), G.T_v0, G.v0_0);
    const float u1 = ffma(float(iu1), G.T_u1, G.u1_0);
    const float u0 = ffma(float(iu0), G.T_u0, G.u0_0);
    const float cs = G.cos_psi, sn = G.sin_psi;
    r.px = fmul(u0, cs);
    r.py = fmul(u0, sn);
    r.pz = u1;
    r.rx = -ffma(v0, cs, sn);
    r.ry = -ffma(v0, sn, -cs);
    r.rz = -v1;
    r.xdriven = fabsf(r.rx) >= fabsf(r.ry);
    const float Tu0_inv = __frcp_rn(G.T_u0);
    if (r.xdriven) {
        r.width = fmul(fmul(0.5f, G.T_u0), fabsf(sn));
        r.trig_inv = __frcp_rn(sn);
        r.inv = __frcp_rn(r.rx);
    } else {
        r.width = fmul(fmul(0.5f, G.T_u0), fabsf(cs));
        r.trig_inv = __frcp_rn(cs);
        r.inv = __frcp_rn(r.ry);
    }
    r.l_phi = fmul(G.T_x, fabsf(r.trig_inv));
    r.fw = fmul(fmul(fmul(0.5f, G.T_x), fabsf(r.trig_inv)), Tu0_inv);
    r.rs = __frsqrt_rn(ffma(v0, v0, ffma(v1, v1, 1.0f)));
    return r;
}

struct PlaneTaps {
    float t;
    int a_min, a_max;  // in-plane voxel index range (x for y-driven, y for x-driven)
    int z_min, z_max;
};

__device__ __forceinline__ void z_range(const petl_geom& G, float z_c, int& z_min, int& z_max)
{
    const float width_z = fmul(0.5f, G.T_u1);
    const float hz = fmul(0.5f, G.T_z);
    const float Tz_inv = __frcp_rn(G.T_z);
    z_min = max(0, int(ceilf(fmul(fsub(fsub(fsub(z_c, width_z), hz), G.z_0), Tz_inv))));
    z_max = min(G.numZ - 1, int(floorf(fmul(fsub(fadd(fadd(z_c, width_z), hz), G.z_0), Tz_inv))));
}

// driving plane y = y(iy) (src/projectors.cu:140-156)
__device__ __forceinline__ PlaneTaps plane_taps_y(const petl_geom& G, const RayGeom& r, int iy)
{
    PlaneTaps p;
    const float y = ffma(float(iy), G.T_x, G.y_0);
    p.t = fmul(fsub(y, r.py), r.inv);
    const float x_c = ffma(p.t, r.rx, r.px);
    const float z_c = ffma(p.t, r.rz, r.pz);
    const float hx = fmul(0.5f, G.T_x);
    const float Tx_inv = __frcp_rn(G.T_x);
    p.a_min = max(0, int(ceilf(fmul(fsub(fsub(fsub(x_c, r.width), hx), G.x_0), Tx_inv))));
    p.a_max = min(G.numX - 1, int(floorf(fmul(fsub(fadd(fadd(x_c, r.width), hx), G.x_0), Tx_inv))));
    z_range(G, z_c, p.z_min, p.z_max);
    return p;
}

// driving plane x = x(ix) (src/projectors.cu:85-101)
__device__ __forceinline__ PlaneTaps plane_taps_x(const petl_geom& G, const RayGeom& r, int ix)
{
    PlaneTaps p;
    const float x = ffma(float(ix), G.T_x, G.x_0);
    p.t = fmul(fsub(x, r.px), r.inv);
    const float y_c = ffma(p.t, r.ry, r.py);
    const float z_c = ffma(p.t, r.rz, r.pz);
    const float hy = fmul(0.5f, G.T_x);
    const float Ty_inv = __frcp_rn(G.T_x);
    p.a_min = max(0, int(ceilf(fmul(fsub(fsub(fsub(y_c, r.width), hy), G.y_0), Ty_inv))));
    p.a_max = min(G.numY - 1, int(floorf(fmul(fsub(fadd(fadd(y_c, r.width), hy), G.y_0), Ty_inv))));
    z_range(G, z_c, p.z_min, p.z_max);
    return p;
}

// u0 footprint of voxel column ix on plane t (y-driven, lines 158-168)
__device__ __forceinline__ float tap_w0_y(const petl_geom& G, const RayGeom& r, float t, int ix, int iu0)
{
    const float x = fsub(ffma(float(ix), G.T_x, G.x_0), fmul(t, r.rx));
    const float c = fmul(fsub(fmul(x, r.trig_inv), G.u0_0), __frcp_rn(G.T_u0));
    return box_overlap(iu0, c, r.fw);
}

// u0 footprint of voxel row iy on plane t (x-driven, lines 103-113)
__device__ __forceinline__ float tap_w0_x(const petl_geom& G, const RayGeom& r, float t, int iy, int iu0)
{
    const float y = fsub(ffma(float(iy), G.T_x, G.y_0), fmul(t, r.ry));
    const float c = fmul(fsub(fmul(y, r.trig_inv), G.u0_0), __frcp_rn(G.T_u0));
    return box_overlap(iu0, c, r.fw);
}

// u1 footprint of voxel slice iz on plane t (lines 104/116-119)
__device__ __forceinline__ float tap_w1(const petl_geom& G, const RayGeom& r, float t, int iz, int iu1)
{
    const float Tu1_inv = __frcp_rn(G.T_u1);
    const float z = fmul(fsub(fsub(ffma(float(iz), G.T_z, G.z_0), fmul(t, r.rz)), G.u1_0), Tu1_inv);
    const float zfw = fmul(fmul(0.5f, G.T_z), Tu1_inv);
    return fmaxf(0.0f, box_overlap(iu1, z, zfw));
}

// The views a call touches: v1 slices [iv1_begin, iv1_end) and, within each,
// the views iv0 = iv0_first + k*iv0_step (ordered subsets use the step).
struct ViewRange {
    int iv1_begin, iv1_end, iv0_first, iv0_step;
    __host__ __device__ int n_v0(int N_v0) const { return iv0_first >= N_v0 ? 0 : (N_v0 - iv0_first + iv0_step - 1) / iv0_step; }
};

// MLEM ratio as the reference's rdivide computes it (src/data_cube.cpp:150-155):
// measured / projected, 0 where the projection is 0.
__device__ __forceinline__ float ratio_rule(float meas, float proj) { return proj == 0.0f ? 0.0f : meas / proj; }

// launchers (projector_general.cu, projector_shear.cu).  meas != nullptr
// stores meas / (P f) (ratio_rule) instead of P f.
int launch_project_general(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                           cudaStream_t st);
int launch_backproject_general(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                               const ViewRange& vr, cudaStream_t st);
int launch_count_nnz(const petl_geom& G, unsigned long long* d_count, cudaStream_t st);
// Split forward projection for any psi with equal voxel height and u1 pitch
// (projector_gsplit.cu); -2 when its layout rules fail (the caller then runs
// launch_project_general).
int project_gsplit(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                   cudaStream_t st);
// Its exact transpose (backprojector_gsplit.cu, adjoint mode); -2 when the
// layout rules fail (the caller then runs launch_backproject_general).
int backproject_gsplit_adjoint(const petl_geom& G, const float* g, float* f, int accumulate, float scale,
                               const ViewRange& vr, cudaStream_t st);
// Backprojection with the reference's semantics for any psi, split into an
// in-plane pass per (v1, u1) slice and a z pass (backprojector_rsplit.cu);
// -2 when its layout rules fail (the caller then runs
// launch_backproject_general).
int backproject_rsplit(const petl_geom& G, const float* g, float* f, int accumulate, float scale,
                       const ViewRange& vr, cudaStream_t st);

}  // namespace petl
