// BF16-storage entry points: volumes and planograms held in bfloat16 (half
// the bytes of FP32), footprints accumulated in FP32.  No reference
// counterpart (the reference stores float32 only); they serve the storage
// precision study and memory-bound serving.  They run the TMA-staged
// shear-warp kernels only, so the geometry must be axis-aligned with voxel
// pitch equal to bin pitch, and the volume rows and planogram rows must be
// multiples of 8 elements (16 bytes); other geometries are refused with an
// error rather than converted behind the caller's back.
#include <cuda_bf16.h>

#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"

namespace petl {
bool shear_eligible(const petl_geom& G);
bool range_ok(const petl_geom& G, const ViewRange& vr);

namespace {

using bf16 = __nv_bfloat16;

int bf16_prologue(const petl_geom* G, const ViewRange& vr, const char* what, shear::TableBuf& tb, cudaStream_t st)
{
    std::string why;
    PETL_REQUIRE(G && geom_valid(G, &why), std::string(what) + ": invalid geometry " + why);
    PETL_REQUIRE(range_ok(*G, vr), std::string(what) + ": invalid view range");
    PETL_REQUIRE(shear_eligible(*G), std::string(what) +
                                         ": BF16 storage needs an axis-aligned planogram (psi = 0) whose bin pitch "
                                         "equals the voxel pitch");
    return shear::make_tables(*G, tb, st);
}

int bf16_result(int rc, const char* what, shear::TableBuf& tb, cudaStream_t st)
{
    cudaFreeAsync(tb.base, st);
    if (rc == shear::kNotApplicable) {
        set_error(std::string(what) +
                  ": BF16 storage needs 16-byte aligned buffers, volume and planogram rows that are multiples of 8 "
                  "elements, N_u0 and numX at most 256 for the backprojection, and slope spreads within the tile "
                  "bounds");
        return -1;
    }
    if (rc == 0) note_path(2);
    return rc;
}

__global__ void k_mlem_update_bf16(bf16* __restrict__ f, const float* __restrict__ d, const float* __restrict__ s,
                                   long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float den = s[i];
        f[i] = __float2bfloat16_rn(__bfloat162float(f[i]) * (den == 0.0f ? 0.0f : d[i] / den));
    }
}

__global__ void k_to_bf16(const float* __restrict__ x, bf16* __restrict__ y, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        y[i] = __float2bfloat16_rn(x[i]);
}

}  // namespace
}  // namespace petl

using namespace petl;

extern "C" {

int petl_project_bf16_dev(const petl_geom* G, const void* f, void* g, int iv1_begin, int iv1_end, int iv0_first,
                          int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(f && g, "project_bf16: null buffer");
    cudaStream_t st = as_stream(stream);
    const ViewRange vr{iv1_begin, iv1_end, iv0_first, iv0_step};
    shear::TableBuf tb;
    int rc = bf16_prologue(G, vr, "project_bf16", tb, st);
    if (rc) return rc;
    rc = shear::project_tma_bf16(*G, static_cast<const bf16*>(f), static_cast<bf16*>(g), vr, nullptr, tb.T, st);
    return bf16_result(rc, "project_bf16", tb, st);
}

int petl_project_ratio_bf16_dev(const petl_geom* G, const void* f, const void* meas, void* ratio, int iv1_begin,
                                int iv1_end, int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(f && meas && ratio, "project_ratio_bf16: null buffer");
    cudaStream_t st = as_stream(stream);
    const ViewRange vr{iv1_begin, iv1_end, iv0_first, iv0_step};
    shear::TableBuf tb;
    int rc = bf16_prologue(G, vr, "project_ratio_bf16", tb, st);
    if (rc) return rc;
    rc = shear::project_tma_bf16(*G, static_cast<const bf16*>(f), static_cast<bf16*>(ratio), vr,
                                 static_cast<const bf16*>(meas), tb.T, st);
    return bf16_result(rc, "project_ratio_bf16", tb, st);
}

int petl_backproject_bf16_dev(const petl_geom* G, const void* g, float* f, int mode, int accumulate, float scale,
                              int iv1_begin, int iv1_end, int iv0_first, int iv0_step, void* stream)
{
    clear_error();
    PETL_REQUIRE(g && f, "backproject_bf16: null buffer");
    PETL_REQUIRE(mode == PETL_BP_REFERENCE || mode == PETL_BP_ADJOINT, "backproject_bf16: unknown mode");
    cudaStream_t st = as_stream(stream);
    const ViewRange vr{iv1_begin, iv1_end, iv0_first, iv0_step};
    shear::TableBuf tb;
    int rc = bf16_prologue(G, vr, "backproject_bf16", tb, st);
    if (rc) return rc;
    rc = shear::backproject_tma_bf16(*G, static_cast<const bf16*>(g), f, mode, accumulate, scale, vr, tb.T, st);
    return bf16_result(rc, "backproject_bf16", tb, st);
}

int petl_to_bf16_dev(const float* x, void* y, long long n, void* stream)
{
    clear_error();
    PETL_REQUIRE(x && y && n >= 0, "to_bf16: invalid arguments");
    if (n == 0) return 0;
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
    k_to_bf16<<<unsigned(blocks), 256, 0, as_stream(stream)>>>(x, static_cast<bf16*>(y), n);
    PETL_LAUNCH_CHECK("to_bf16");
    return 0;
}

int petl_mlem_update_bf16_dev(void* f, const float* d, const float* sens, long long n, void* stream)
{
    clear_error();
    PETL_REQUIRE(f && d && sens && n >= 0, "mlem_update_bf16: invalid arguments");
    if (n == 0) return 0;
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
    k_mlem_update_bf16<<<unsigned(blocks), 256, 0, as_stream(stream)>>>(static_cast<bf16*>(f), d, sens, n);
    PETL_LAUNCH_CHECK("mlem_update_bf16");
    return 0;
}

}  // extern "C"
