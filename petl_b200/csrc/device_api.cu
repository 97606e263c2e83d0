// Device-pointer entry points (petl_device.h) and kernel dispatch.
//
// The projector entry points choose between the shear kernels of
// projector_shear.cu (axis-aligned planograms whose voxel pitch equals the bin
// pitch: every benchmark configuration) and the general kernels of
// projector_general.cu (any orientation and pitch).  Both compute the same
// operator; the dispatch only changes how fast.
#include <cmath>
#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"

namespace petl {
int pfdr(const petl_geom& G, const float* g, float* g_reb, cudaStream_t st);
int ramp(const petl_geom& G, float* g_reb, int apply_weight, cudaStream_t st);
int launch_gaussian(float* f, int N1, int N2, int N3, float FWHM, int numDims, cudaStream_t st);

// shear fast path (projector_shear.cu)
bool shear_eligible(const petl_geom& G);
int launch_project_shear(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                         cudaStream_t st);
int launch_backproject_shear(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                             const ViewRange& vr, cudaStream_t st);

int g_dispatch = -1;  // -1: read PETL_FORCE_GENERAL once

int dispatch_mode()
{
    if (g_dispatch < 0) {
        const char* e = getenv("PETL_FORCE_GENERAL");
        g_dispatch = (e && e[0] == '1') ? 1 : 0;
    }
    return g_dispatch;
}

bool use_shear(const petl_geom& G) { return dispatch_mode() != 1 && shear_eligible(G); }

thread_local int t_last_path = -1;
void note_path(int path) { t_last_path = path; }

bool range_ok(const petl_geom& G, const ViewRange& vr)
{
    return vr.iv1_begin >= 0 && vr.iv1_end <= G.N_v1 && vr.iv1_begin <= vr.iv1_end && vr.iv0_first >= 0 &&
           vr.iv0_step >= 1;
}

// ---------------------------------------------------------------------------
// psi = 90 degrees (the second planogram of PET/X, src/petx_server.py:9-10).
// The reference takes its x-driven branch there (src/projectors.cu:77-130):
// the ray through bin (u0, u1) of view (v0, v1) crosses the plane at x in
// y = u0 + v0 x, z = u1 + v1 x, which is the psi = 0 (y-driven) ray of
// plane t = -x on a volume whose axes are exchanged: x' = y, y' = -x.  The
// projection is therefore the shear-warp projection of the transposed,
// flipped volume f'[z][nx-1-ix][iy] = f[z][iy][ix] under the psi = 0
// geometry with those axes (equal pitch in x and y, which the volume has),
// and the backprojection is the flip of the shear-warp backprojection.  The
// reference evaluates cos(pi/2) in float (-4.4e-8, not 0), which moves its
// ray coordinates by parts in 1e8: the two agree to rounding.
// ---------------------------------------------------------------------------
namespace {

bool psi90(const petl_geom& G)
{
    return std::fabs(G.cos_psi) < 1e-6f && G.sin_psi == 1.0f;
}

petl_geom transposed(const petl_geom& G)
{
    petl_geom T = G;
    T.cos_psi = 1.0f;
    T.sin_psi = 0.0f;
    T.numX = G.numY;
    T.numY = G.numX;
    T.x_0 = G.y_0;
    T.y_0 = -(G.x_0 + float(G.numX - 1) * G.T_x);
    return T;
}

// dir 0: out[z][nx-1-ix][iy] = in[z][iy][ix] (in: nz x ny x nx)
// dir 1: out[z][iy][ix] (+)= in[z][nx-1-ix][iy] (in: nz x nx x ny)
__global__ void __launch_bounds__(256)
k_flip_transpose(const float* __restrict__ in, float* __restrict__ out, int nx, int ny, int dir, int accumulate)
{
    __shared__ float tile[32][33];
    const int z = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    if (dir == 0) {
        const int ix0 = blockIdx.x * 32, iy0 = blockIdx.y * 32;
        for (int r = ty; r < 32; r += 8) {
            const int iy = iy0 + r, ix = ix0 + tx;
            if (iy < ny && ix < nx) tile[r][tx] = in[(size_t(z) * ny + iy) * nx + ix];
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            const int ix = ix0 + r, iy = iy0 + tx;  // out row nx-1-ix, column iy
            if (iy < ny && ix < nx) out[(size_t(z) * nx + (nx - 1 - ix)) * ny + iy] = tile[tx][r];
        }
    } else {
        const int iy0 = blockIdx.x * 32, r0 = blockIdx.y * 32;  // in: rows r = nx-1-ix, columns iy
        for (int r = ty; r < 32; r += 8) {
            const int row = r0 + r, iy = iy0 + tx;
            if (row < nx && iy < ny) tile[r][tx] = in[(size_t(z) * nx + row) * ny + iy];
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            const int iy = iy0 + r, row = r0 + tx, ix = nx - 1 - row;
            if (row < nx && iy < ny) {
                const size_t o = (size_t(z) * ny + iy) * nx + ix;
                const float v = tile[tx][r];
                out[o] = accumulate ? out[o] + v : v;
            }
        }
    }
}

int flip_transpose(const float* in, float* out, const petl_geom& G, int dir, int accumulate, cudaStream_t st)
{
    const dim3 block(32, 8);
    const dim3 grid = dir == 0 ? dim3(ceil_div(G.numX, 32), ceil_div(G.numY, 32), unsigned(G.numZ))
                               : dim3(ceil_div(G.numY, 32), ceil_div(G.numX, 32), unsigned(G.numZ));
    k_flip_transpose<<<grid, block, 0, st>>>(in, out, G.numX, G.numY, dir, accumulate);
    PETL_LAUNCH_CHECK("flip_transpose");
    return 0;
}

bool use_psi90_shear(const petl_geom& G)
{
    return dispatch_mode() != 1 && psi90(G) && G.T_x == G.T_u0 && G.numZ <= 65535 && shear_eligible(transposed(G));
}

}  // namespace

int project_range(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                  cudaStream_t st)
{
    std::string why;
    PETL_REQUIRE(geom_valid(&G, &why), "project: " + why);
    PETL_REQUIRE(f && g && range_ok(G, vr), "project: invalid arguments");
    if (vr.iv1_begin == vr.iv1_end || vr.iv0_first >= G.N_v0) return 0;
    if (use_shear(G)) return launch_project_shear(G, f, g, vr, meas, st);
    if (use_psi90_shear(G)) {
        const petl_geom T = transposed(G);
        float* ft = nullptr;
        PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&ft), sizeof(float) * size_t(G.numX) * G.numY * G.numZ, st));
        int rc = flip_transpose(f, ft, G, 0, 0, st);
        if (!rc) rc = launch_project_shear(T, ft, g, vr, meas, st);
        cudaFreeAsync(ft, st);
        return rc;
    }
    if (dispatch_mode() == 0) {
        const int rc = project_gsplit(G, f, g, vr, meas, st);
        if (rc != -2) {  // applied (-2: its layout rules fail)
            note_path(3);
            return rc;
        }
    }
    note_path(0);
    return launch_project_general(G, f, g, vr, meas, st);
}

int backproject_range(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                      const ViewRange& vr, cudaStream_t st)
{
    std::string why;
    PETL_REQUIRE(geom_valid(&G, &why), "backproject: " + why);
    PETL_REQUIRE(f && g && range_ok(G, vr), "backproject: invalid arguments");
    PETL_REQUIRE(mode == PETL_BP_REFERENCE || mode == PETL_BP_ADJOINT, "backproject: unknown mode");
    if (use_shear(G)) return launch_backproject_shear(G, g, f, mode, accumulate, scale, vr, st);
    if (use_psi90_shear(G)) {
        const petl_geom T = transposed(G);
        float* bt = nullptr;
        PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&bt), sizeof(float) * size_t(G.numX) * G.numY * G.numZ, st));
        int rc = launch_backproject_shear(T, g, bt, mode, 0, scale, vr, st);
        if (!rc) rc = flip_transpose(bt, f, G, 1, accumulate, st);
        cudaFreeAsync(bt, st);
        return rc;
    }
    if (dispatch_mode() == 0) {
        const int rc = mode == PETL_BP_ADJOINT ? backproject_gsplit_adjoint(G, g, f, accumulate, scale, vr, st)
                                               : backproject_rsplit(G, g, f, accumulate, scale, vr, st);
        if (rc != -2) {
            note_path(3);
            return rc;
        }
    }
    note_path(0);
    return launch_backproject_general(G, g, f, mode, accumulate, scale, vr, st);
}

int fbp(const petl_geom& G, const float* g, float* f, int accumulate, cudaStream_t st, float* host_rebinned_out)
{
    std::string why;
    PETL_REQUIRE(geom_valid(&G, &why), "FBP: " + why);
    petl_geom Gr = G;
    const size_t nreb = size_t(G.N_v0) * G.N_u1 * G.N_u0;
    float* reb = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&reb), sizeof(float) * nreb, st));
    int rc = 0;
    if (G.N_v1 > 1) {
        // PETL::doFBP -> doPFDR, then the rebinned geometry (src/petl.cpp:379-380)
        rc = pfdr(G, g, reb, st);
        Gr.N_v1 = 1;
        Gr.v1_0 = 0.0f;
    } else {
        cudaError_t e = cudaMemcpyAsync(reb, g, sizeof(float) * nreb, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            set_error(std::string("FBP: ") + cudaGetErrorString(e));
            rc = int(e);
        }
    }
    if (!rc) rc = ramp(Gr, reb, 1, st);
    if (!rc && host_rebinned_out) {
        cudaError_t e = cudaMemcpyAsync(host_rebinned_out, reb, sizeof(float) * nreb, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = int(e);
    }
    // FBPweight scale T_v0*T_u0/voxelWidth (src/petl.cpp:254-259), float
    const float scale = Gr.T_v0 * Gr.T_u0 / Gr.T_x;
    if (!rc) rc = backproject_range(Gr, reb, f, PETL_BP_REFERENCE, accumulate, scale, ViewRange{0, 1, 0, 1}, st);
    cudaFreeAsync(reb, st);
    return rc;
}

}  // namespace petl

using namespace petl;

extern "C" {

int petl_last_projector_path(void) { return t_last_path; }

int petl_set_dispatch(int mode)
{
    // 0: the fastest kernels that apply; 1: always the general kernels;
    // 2: shear kernels without TMA staging where the shear path applies;
    // 3: TMA-staged shear kernels with the fused (single-kernel) forward
    if (mode < 0 || mode > 3) return -1;
    g_dispatch = mode;
    return 0;
}

int petl_project_dev(const petl_geom* G, const float* f, float* g, int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(G, "project: null geometry");
    return project_range(*G, f, g, ViewRange{0, G->N_v1, iv0_first, iv0_step}, nullptr, as_stream(stream));
}

int petl_project_range_dev(const petl_geom* G, const float* f, float* g, int iv1_begin, int iv1_end, int iv0_first,
                           int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(G, "project: null geometry");
    return project_range(*G, f, g, ViewRange{iv1_begin, iv1_end, iv0_first, iv0_step}, nullptr, as_stream(stream));
}

int petl_project_ratio_dev(const petl_geom* G, const float* f, const float* meas, float* ratio, int iv1_begin,
                           int iv1_end, int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(G && meas, "project_ratio: invalid arguments");
    return project_range(*G, f, ratio, ViewRange{iv1_begin, iv1_end, iv0_first, iv0_step}, meas, as_stream(stream));
}

int petl_backproject_dev(const petl_geom* G, const float* g, float* f, int mode, int accumulate, float scale,
                         int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(G, "backproject: null geometry");
    return backproject_range(*G, g, f, mode, accumulate, scale, ViewRange{0, G->N_v1, iv0_first, iv0_step},
                             as_stream(stream));
}

int petl_backproject_range_dev(const petl_geom* G, const float* g, float* f, int mode, int accumulate, float scale,
                               int iv1_begin, int iv1_end, int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(G, "backproject: null geometry");
    return backproject_range(*G, g, f, mode, accumulate, scale, ViewRange{iv1_begin, iv1_end, iv0_first, iv0_step},
                             as_stream(stream));
}

int petl_project_nnz_dev(const petl_geom* G, double* nnz_host, void* stream)
{
    clear_error();
    std::string why;
    PETL_REQUIRE(G && nnz_host && geom_valid(G, &why), "project_nnz: invalid arguments " + why);
    cudaStream_t st = as_stream(stream);
    unsigned long long* d = nullptr;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(&d), sizeof(unsigned long long), st));
    PETL_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), st));
    int rc = launch_count_nnz(*G, d, st);
    unsigned long long h = 0;
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error(std::string("project_nnz: ") + cudaGetErrorString(e));
            rc = int(e);
        }
    }
    cudaFreeAsync(d, st);
    *nnz_host = double(h);
    return rc;
}

int petl_pfdr_dev(const petl_geom* G, const float* g, float* g_reb, void* stream)
{
    clear_error();
    std::string why;
    PETL_REQUIRE(G && g && g_reb && geom_valid(G, &why), "PFDR: invalid arguments " + why);
    return pfdr(*G, g, g_reb, as_stream(stream));
}

int petl_ramp_dev(const petl_geom* G, float* g_reb, int apply_weight, void* stream)
{
    clear_error();
    std::string why;
    PETL_REQUIRE(G && g_reb && geom_valid(G, &why), "ramp: invalid arguments " + why);
    return ramp(*G, g_reb, apply_weight, as_stream(stream));
}

int petl_fbp_dev(const petl_geom* G, const float* g, float* f, int accumulate, void* stream)
{
    clear_error();
    PETL_REQUIRE(G && g && f, "FBP: invalid arguments");
    return fbp(*G, g, f, accumulate, as_stream(stream), nullptr);
}

int petl_gaussian_filter_dev(float* f, int N1, int N2, int N3, float FWHM, int numDims, void* stream)
{
    clear_error();
    PETL_REQUIRE(f && N1 > 0 && N2 > 0 && N3 > 0, "gaussian_filter: invalid arguments");
    return launch_gaussian(f, N1, N2, N3, FWHM, numDims, as_stream(stream));
}

}  // extern "C"
