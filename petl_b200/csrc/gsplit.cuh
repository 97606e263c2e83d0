// Pieces shared by the split projector kernels for any psi: the forward
// (projector_gsplit.cu) and its exact adjoint (backprojector_gsplit.cu).
#pragma once
#include <cmath>
#include <cstddef>

#include "common.cuh"
#include "projector.cuh"

namespace petl {

// Bytes of FP32 scratch one call may hold (its chunk of views).
inline size_t gsplit_scratch_budget() { return size_t(5) << 30; }

// The ray parameter of the lane's ray on driving plane p (y = const for a
// y-driven view, x = const for an x-driven one), as plane_taps_x/_y form it.
__device__ __forceinline__ float plane_t(const petl_geom& G, const RayGeom& r, int p)
{
    return r.xdriven ? fmul(fsub(ffma(float(p), G.T_x, G.x_0), r.px), r.inv)
                     : fmul(fsub(ffma(float(p), G.T_x, G.y_0), r.py), r.inv);
}

// plain x/y transpose of every z slice: out[z][x][y] = in[z][y][x] (nx, ny of
// the input); with add, out += in transposed times scale
__global__ void k_transpose_xy(const float* __restrict__ in, float* __restrict__ out, int nx, int ny);

// host: the ray quantities of view iv0 as ray_geom computes them
struct HostView {
    bool xd;
    double inv, pscale;  // 1/r_p and |sin| or |cos| (p-coordinate of u0 = u0 * pscale)
};

inline HostView host_view(const petl_geom& G, int iv0)
{
    const float v0 = std::fmaf(float(iv0), G.T_v0, G.v0_0);
    const float rx = -std::fmaf(v0, G.cos_psi, G.sin_psi), ry = -std::fmaf(v0, G.sin_psi, -G.cos_psi);
    HostView h;
    h.xd = std::fabs(rx) >= std::fabs(ry);
    h.inv = 1.0 / double(h.xd ? rx : ry);
    h.pscale = std::fabs(double(h.xd ? G.cos_psi : G.sin_psi));
    return h;
}

}  // namespace petl
