// Shift tables shared by the shear-warp projector kernels (projector_shear.cu,
// projector_shear_tma.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "projector.cuh"

namespace petl {
namespace shear {

struct Shift {
    int d;    // integer part of the shift
    float w;  // fractional weight of the second tap
};

struct Tables {
    Shift* xt;      // [N_v0][N_y]
    Shift* zt;      // [N_v1][N_y]
    float* S;       // [N_v1][N_v0]  l_phi * rsqrt(1 + v0^2 + v1^2)
    int2* zvis;     // [N_v1][N_y]   voxel-centre visible iz range (reference backprojector)
    int2* ub0;      // [N_v0]        visible iu0 range of the forward masks
    int2* ub1;      // [N_v1]        visible iu1 range of the forward masks
};

// The split kernels (projector_split.cu, backprojector_split.cu) move a
// volume-sized scratch array per view; with fewer slopes than this a call
// takes the single-pass kernels instead.
constexpr int kSplitMinSlopes = 10;

// The volumes (or planograms) one launch of a split kernel serves: a plain
// call has one member; a batched call has up to kMaxMembers requests of the
// same geometry, each with its own buffers and its own view subset (first
// view, the common view step).  Member b's views v = 0 .. nv[b] - 1 are view
// iv0 = first[b] + v * step of the geometry and occupy the scratch view
// slots b * nvm + v.
constexpr int kMaxMembers = 8;
struct Members {
    int nb = 1;                         // members
    int nvm = 0;                        // view slots per member (the largest nv)
    int first[kMaxMembers] = {};        // first view of each member in this launch
    int nv[kMaxMembers] = {};           // views of each member in this launch
    const void* in[kMaxMembers] = {};   // volume (forward) or planogram (backward)
    void* out[kMaxMembers] = {};        // planogram (forward) or volume (backward)
    const void* meas[kMaxMembers] = {}; // measured planogram of the forward's MLEM ratio, or null
};

// member b's entry of a per-member parameter array, by selects (a dynamic
// index would copy the kernel's parameter block to local memory); kernels
// compiled for one member (NM = 1) read entry 0
template <int NM = kMaxMembers, class T>
__device__ __forceinline__ T member_pick(const T (&a)[kMaxMembers], int b)
{
    T v = a[0];
#pragma unroll
    for (int i = 1; i < NM; i++)
        if (b == i) v = a[i];
    return v;
}

// per-call table workspace (stream-ordered)
struct TableBuf {
    void* base = nullptr;
    Tables T{};
    size_t bytes = 0;
};

int make_tables(const petl_geom& G, TableBuf& tb, cudaStream_t st);

// Largest |y| of the volume's plane centres.
inline double plane_ymax(const petl_geom& G)
{
    return std::fmax(std::fabs(double(G.y_0)), std::fabs(double(G.y_0) + (G.numY - 1) * double(G.T_x)));
}

// Upper bound on the difference of the integer z shifts of slopes (or planes)
// n steps apart: the exact shifts differ by at most n * step, their floors by
// at most floor(n * step) + 1 (with a relative margin for the float inputs).
inline int shift_spread(int n, double step) { return int(std::floor(double(n) * step * (1.0 + 1e-6))) + 1; }

// Bytes of FP32 scratch one split projection call may hold (its chunk of
// views): PETL_SPLIT_SCRATCH_MB, else 5 GiB, at most an eighth of the
// device's memory.
size_t split_scratch_budget();

// Called once per chunk of views of a split projection, on the host while
// the chunk's work is enqueued: after the forward's kernels of the chunk
// (to start copying its planogram views out) or before the backward's (to
// make the stream wait for its planogram views).  vi0 is the chunk's first
// view index in the call's view range, nvc its view count.
struct ChunkHook {
    void (*fn)(void* ctx, int vi0, int nvc) = nullptr;
    void* ctx = nullptr;
};

// Split forward projection (projector_split.cu): an x-shift pass per chunk of
// views into FP32 scratch, then a z-tap kernel fed by a TMA ring.  Same
// operator and the same float operations in the same order as project_tma.
// chunk_cap > 0 bounds the views per chunk.  kNotApplicable when the layout
// rules or the scratch allocation fail.
int project_split(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                  const Tables& T, cudaStream_t st, int chunk_cap = 0, const ChunkHook* hook = nullptr);
int project_split_bf16(const petl_geom& G, const __nv_bfloat16* f, __nv_bfloat16* g, const ViewRange& vr,
                       const __nv_bfloat16* meas, const Tables& T, cudaStream_t st);
// Split backprojection (backprojector_split.cu): a z-gather kernel per chunk
// of views into FP32 scratch, then an x-gather pass that sums the views into
// the volume.  Same operator and the same float operations in the same order
// as backproject_tma; kNotApplicable when the layout rules or the scratch
// allocation fail.
int backproject_split(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                      const ViewRange& vr, const Tables& T, cudaStream_t st, int chunk_cap = 0,
                      const ChunkHook* hook = nullptr);
int backproject_split_bf16(const petl_geom& G, const __nv_bfloat16* g, float* f, int mode, int accumulate,
                           float scale, const ViewRange& vr, const Tables& T, cudaStream_t st);
// The same for the members of M (FP32): one launch of each split kernel
// serves all of them, every member's result equal bit for bit to its own
// call.  vr gives the slopes and the view step; the members' first views and
// view counts are in M.  kNotApplicable when the split kernels do not apply
// or the members' views do not fit one chunk of scratch.
int project_split_members(const petl_geom& G, const Members& M, const ViewRange& vr, const Tables& T,
                          cudaStream_t st);
int backproject_split_members(const petl_geom& G, const Members& M, int mode, int accumulate, float scale,
                              const ViewRange& vr, const Tables& T, cudaStream_t st);

// Bytes of the shift tables of G (make_tables' allocation).
size_t table_bytes(const petl_geom& G);

// The fastest shear kernels that apply, with caller-held tables (TMA-staged,
// else first generation).  The geometry must pass shear_eligible.
int project_with(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                 const Tables& T, cudaStream_t st);
int backproject_with(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                     const ViewRange& vr, const Tables& T, cudaStream_t st);

// Return value of the TMA launchers when the geometry or the buffers do not
// fit their layout rules; the caller then uses the first-generation kernels.
constexpr int kNotApplicable = -2;

// Projection of all views of G by the split kernels in chunks of at most
// chunk_cap views, with the shift tables built here and `hook` called per
// chunk; kNotApplicable when the split kernels do not apply (the caller then
// projects without chunk hooks).
int project_chunked(const petl_geom& G, const float* f, float* g, int chunk_cap, const ChunkHook& hook,
                    cudaStream_t st);
int backproject_chunked(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                        int chunk_cap, const ChunkHook& hook, cudaStream_t st);

// TMA-staged kernels (projector_shear_tma.cu).  They compute the same
// operator as the first-generation kernels of projector_shear.cu.
int project_tma(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                const Tables& T, cudaStream_t st);
int backproject_tma(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                    const ViewRange& vr, const Tables& T, cudaStream_t st);
// BF16 storage (volume and planogram in bfloat16, FP32 arithmetic; the
// backprojection writes an FP32 volume).  Same layout rules with 2-byte
// elements.
int project_tma_bf16(const petl_geom& G, const __nv_bfloat16* f, __nv_bfloat16* g, const ViewRange& vr,
                     const __nv_bfloat16* meas, const Tables& T, cudaStream_t st);
int backproject_tma_bf16(const petl_geom& G, const __nv_bfloat16* g, float* f, int mode, int accumulate, float scale,
                         const ViewRange& vr, const Tables& T, cudaStream_t st);

}  // namespace shear

// Projector kernel choice (petl_set_dispatch): 0 automatic, 1 general kernels
// only, 2 shear kernels without TMA staging where the shear path applies, 3
// TMA-staged shear kernels with the fused forward instead of the split one.
int dispatch_mode();
// Records which projector kernels the calling thread used last
// (petl_last_projector_path): 0 general, 1 shear, 2 TMA-staged shear.
void note_path(int path);

}  // namespace petl
