// Shear-warp projector kernels for axis-aligned planograms (placeholder:
// the dispatch falls back to the general kernels until these are enabled).
#include "common.cuh"
#include "projector.cuh"

namespace petl {

bool shear_eligible(const petl_geom&) { return false; }

int launch_project_shear(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                         cudaStream_t st)
{
    return launch_project_general(G, f, g, vr, meas, st);
}

int launch_backproject_shear(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                             const ViewRange& vr, cudaStream_t st)
{
    return launch_backproject_general(G, g, f, mode, accumulate, scale, vr, st);
}

}  // namespace petl
