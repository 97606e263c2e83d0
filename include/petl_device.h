/*
 * petl_device.h -- device-resident entry points of libpetl.so (B200 build).
 *
 * These have no single counterpart in the reference: the reference C ABI
 * (petl.h) copies host arrays to the GPU and back inside every call
 * (src/projectors.cu:379-497, src/cuda_utils.cu:1146-1361).  The functions
 * here take DEVICE pointers and a CUDA stream (passed as void*), keep no
 * hidden state between calls except cached per-device scratch, and are what
 * the reference-compatible entry points of petl.h call after staging host
 * data.  Each one names the reference routine whose result it reproduces.
 *
 * Layouts: planogram float32 [N_v1][N_v0][N_u1][N_u0], volume float32
 * [numZ][numY][numX], rebinned planogram [N_v0][N_u1][N_u0] (one v1 slice).
 * Return value: 0 on success, nonzero on error; petl_last_error() gives the
 * message for the calling thread.
 */
#ifndef PETL_B200_PETL_DEVICE_H
#define PETL_B200_PETL_DEVICE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One planogram together with the volume it projects to.  Lengths are the
 * HALF lengths the reference stores internally (src/planogram.h:41-51), psi
 * in radians, start values are the coordinates of sample 0. */
typedef struct petl_geom {
    float psi, R, L, H, v_m0, v_m1;
    int   N_v1, N_v0, N_u1, N_u0;
    float T_v1, T_v0, T_u1, T_u0;
    float v1_0, v0_0, u1_0, u0_0;
    float cos_psi, sin_psi;
    int   numX, numY, numZ;
    float T_x, T_z;            /* voxelWidth (x and y), voxelHeight (z) */
    float x_0, y_0, z_0;       /* coordinates of voxel (0,0,0) */
} petl_geom;

/* Backprojector semantics. */
enum {
    PETL_BP_REFERENCE = 0, /* the reference backprojector's visibility rules
                              (src/projectors.cu:240-377) with exact weights */
    PETL_BP_ADJOINT   = 1  /* the exact transpose of petl_project_dev */
};

const char* petl_last_error(void);
int petl_version(void);
/* Number of CUDA kernels this library has launched in this process. */
unsigned long long petl_launch_count(void);

/* planogram::init (src/planogram.cpp:143-186) with the C-ABI conventions of
 * add_planogram (src/petl_c_interface.cpp:216-219): psi in degrees, D/L/H
 * full lengths. */
int petl_geom_init(petl_geom* G, float psi_deg, float D, float L, float H, float v_m0, float v_m1, float T);
/* parameters::set_volume + x_0/y_0/z_0 (src/parameters.cpp:250-284). */
int petl_geom_set_volume(petl_geom* G, int numX, int numY, int numZ, float voxelWidth, float voxelHeight,
                         float offsetX, float offsetY, float offsetZ);
/* optimalFFTsize (src/vector_ops.cpp:481-505). */
int petl_optimal_fft_size(int N);

/* The currently selected model's planogram `which` (and its volume, when the
 * volume is defined) as set through the petl.h setters. */
int petl_model_geometry(int which, petl_geom* out);
/* Copies between a host array and device memory on `stream`, returning once
 * the copy is complete; pageable host arrays are staged through the
 * library's pinned buffers (much faster than the driver's own pageable
 * copies), pinned ones copied directly.  0 on success. */
int petl_copy_to_host(void* host, const void* dev, long long bytes, void* stream);
int petl_copy_to_device(void* dev, const void* host, long long bytes, void* stream);

/* The solids of the selected model's phantom (modules == 0) or detector-module
 * model (modules != 0): copies up to capacity of them into out (may be null)
 * and returns how many there are.  The struct is declared below. */
struct petl_solid;
int petl_model_solids(int modules, struct petl_solid* out, int capacity);

/* Kernel dispatch for the projectors: 0 (default) uses the shear-warp
 * kernels for axis-aligned, equal-pitch geometries (TMA-staged where the
 * layout allows) and the general kernels otherwise; 1 always uses the
 * general kernels; 2 uses the shear-warp kernels without TMA staging where
 * the shear path applies; 3 uses the TMA-staged shear-warp kernels with the
 * single-kernel forward instead of the split forward (x-shift pass into
 * scratch + z-tap kernel).  All compute the same operator. */
int petl_set_dispatch(int mode);
/* Which projector kernels the calling thread's last projector call used:
 * 0 general, 1 shear-warp, 2 TMA-staged shear-warp, 3 the split kernels
 * for any psi (forward, reference-semantics or exact-adjoint
 * backprojection; two passes through scratch); -1 before any call. */
int petl_last_projector_path(void);

/* List-mode binning (src/binning.cpp:614-790 with src/planogram.cpp:113-141):
 * the coincidences blue[i], pink[i] (xyz in mm, i < n, device arrays of 3n
 * floats) are added to the planogram g of G.  linear != 0: bilinear weights
 * in (u1, u0), the reference's binning; else the nearest bin.  chest_wall !=
 * 0: z is measured from the panels' bottom edge (u1 shifted by -H), the
 * reference's list-mode origin.  Accumulates into g (zero it first for the
 * reference's bin, which overwrites).  Deposits are atomic adds, so sums of
 * fractional weights may differ in the last bits from run to run. */
int petl_bin_events_dev(const petl_geom* G, const float* blue, const float* pink, long long n, float* g,
                        int linear, int chest_wall, void* stream);

/* Solid-angle correction of one planogram on the device
 * (src/planogram.cpp:262-302): projection (iv1, iv0) is multiplied by
 * 2 pi (1 + v0^2 + v1^2)^1.5 / (T_v1 T_v0), or by its inverse (the
 * solid-angle model) when do_inverse != 0.  Needs the planogram only. */
int petl_solid_angle_dev(const petl_geom* G, float* g, int do_inverse, void* stream);

/* PETL::apply_corrections on one planogram on the device (src/petl.cpp:
 * 163-192, src/median_filter.cu): g = g / r (0 where r == 0), then per
 * projection, with t = threshold * median of the projection's r: bins outside
 * the field of view -> 0; bins with r < t -> the median of the 5x5 window's
 * divided values above t (edges clamped; 0 if none); other bins keep g / r.
 * Windows read the divided values before any in-fill. */
int petl_apply_corrections_dev(const petl_geom* G, float* g, const float* r, float threshold, void* stream);

/* One analytic solid of a phantom or of the detector-module model
 * (src/phantom.h:23-57, src/analytic_ray_tracing_gpu.cuh:27-39).  type:
 * 0 ellipsoid, 1 parallelepiped, 2/3/4 cylinder along x/y/z, 5/6/7 cone
 * along x/y/z.  centers/radii are the ray tracer's form (cones rewritten to
 * a unit-slope cone and its axial clip range clip_cone, src/phantom.cpp:
 * 594-638); given_c/given_r keep the values as given (the voxelizer
 * rebuilds cones from them, src/phantom.cpp:118-121).  clip planes are
 * (n, d) with n . x >= d kept. */
typedef struct petl_solid {
    int type;
    float centers[3], radii[3];
    float val;
    float A[9];
    float clip[6][4];
    int rotated, num_clip;
    float clip_cone[2];
    float given_c[3], given_r[3];
} petl_solid;

/* geometricObject::init (src/phantom.cpp:535-640): 0, or -1 for a bad type
 * or a null c / r.  A and clip may be null. */
int petl_solid_init(petl_solid* s, int type, const float* c, const float* r, float val, const float* A,
                    const float* clip);

/* phantom::scale_phantom on n solids (src/phantom.cpp:1120-1141). */
void petl_solids_scale(petl_solid* s, int n, float sx, float sy, float sz);

/* phantom::voxelize (src/phantom.cpp:105-335) on the device: the solids in
 * order, each one replacing the voxel values inside it (oversampling 1) or
 * blending toward its value by the fraction of 1..5^3 sub-samples inside.
 * f is [numZ][numY][numX]; x_0/y_0/z_0 are the coordinates of voxel 0. */
int petl_voxelize_dev(const petl_solid* solids, int n, float* f, int numX, int numY, int numZ, float voxelWidth,
                      float voxelHeight, float x_0, float y_0, float z_0, int oversampling, void* stream);

/* Analytic ray tracing of a planogram through n solids
 * (src/analytic_ray_tracing_gpu.cu:693-846, rayTrace_gpu): per bin the
 * sum of value x length of the intervals of the bin's line that each solid
 * (the last one covering an interval) occupies, in the reference's
 * parameterisation (lengths over 1 + v0^2 + v1^2), averaged over an
 * oversampling^2 grid of lines (oversampling odd, 1..11); stopping_power != 0
 * gives (1 - exp(-forward)) (1 - exp(-backward)) of the two half-lines
 * instead.  Bins outside the field of view are 0. */
int petl_ray_trace_dev(const petl_geom* G, const petl_solid* solids, int n, float* g, int oversampling,
                       int stopping_power, void* stream);

/* Error word written by kernels whose waits on asynchronous copies are
 * bounded: nonzero if a wait gave up (the call's result is then invalid).
 * Reading it synchronizes the device and clears it.  -1 if it cannot be
 * read.  The reference-compatible calls (project, backproject, FBP) read it
 * after their own synchronisation and return false when it is set; callers
 * of the stream-ordered entry points here read it themselves. */
int petl_device_error_flag(void);

/* Failure-path hook; no counterpart in the reference.  The projector and
 * PFDR kernels' waits on staged data give up after 2^22 polls: they set the error
 * word, drain their copies in flight (with the full bound) and return
 * without writing.  With on != 0 every such wait of the kernels launched
 * afterwards gives up before polling, which drives that path without a
 * fault or a hang; on == 0 restores the bound.  Process-wide, read when a
 * launch is built. */
int petl_force_wait_timeout(int on);

/* Allocation failure injection; no counterpart in the reference (whose
 * calls leak their device buffers when a cudaMalloc fails).  Every scratch
 * allocation of this library (device buffers of the reference-compatible
 * calls, projector tables and scratch, reductions) comes from one stream-
 * ordered pool per device.  petl_inject_alloc_failure(n) makes the n-th
 * allocation from now fail once as out of memory (n <= 0 disarms);
 * petl_scratch_alloc_count() counts the allocations made so far;
 * petl_scratch_in_use() gives the bytes of the current device's pool held by
 * live allocations (after a synchronisation: 0 when no call is running), -1
 * if it cannot be read. */
int petl_inject_alloc_failure(long long n);
long long petl_scratch_alloc_count(void);
long long petl_scratch_in_use(void);

/* Forward SF projection (src/projectors.cu:11-238).  Computes the views
 * iv0 = iv0_first + k*iv0_step (k = 0.., iv0 < N_v0) of every v1 slice and
 * writes them into the full-size planogram g; other views are untouched.
 * iv0_first = 0, iv0_step = 1 is the whole planogram. */
int petl_project_dev(const petl_geom* G, const float* f, float* g, int iv0_first, int iv0_step, void* stream);

/* Backprojection (src/projectors.cu:240-377, summed over v1 as
 * backproject_SF does).  Only views iv0 = iv0_first + k*iv0_step contribute.
 * f = accumulate ? f + scale*P^T g : scale*P^T g. */
int petl_backproject_dev(const petl_geom* G, const float* g, float* f, int mode, int accumulate, float scale,
                         int iv0_first, int iv0_step, void* stream);

/* Allocation-free forward projection of every view; no counterpart in the
 * reference.  For callers that must not allocate device memory while they
 * run (a real-time acquisition thread that cannot block on the allocator, a
 * program whose own pool owns the GPU's memory).  It computes the same
 * projection as petl_project_dev but keeps its scratch tables in a fixed
 * 4 MiB device array that every GPU loading the library holds until exit,
 * and calls no cudaMalloc/cudaFree or allocating library routine.  A
 * geometry whose tables exceed 4 MiB is rejected with an error (nonzero
 * return, message in petl_last_error()).  All calls on one device share the
 * array, so calls that overlap on the GPU race; each call rewrites the
 * tables it reads, so no clearing is needed.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture.  With
 * CUDA's lazy module loading (the default), the first call of this library
 * on a device -- this one or any other -- loads the library's device code
 * on that device, which allocates device memory (the 4 MiB array among it):
 * make one call during set-up, before the code that must not allocate runs.
 * petl_set_dispatch(1) makes it run the general kernel, which needs no
 * tables. */
int petl_project_noalloc_dev(const petl_geom* G, const float* f, float* g, void* stream);

/* Same as petl_project_dev restricted to the v1 slices [iv1_begin, iv1_end). */
int petl_project_range_dev(const petl_geom* G, const float* f, float* g, int iv1_begin, int iv1_end, int iv0_first,
                           int iv0_step, void* stream);
/* Same as petl_backproject_dev restricted to the v1 slices [iv1_begin, iv1_end). */
int petl_backproject_range_dev(const petl_geom* G, const float* g, float* f, int mode, int accumulate, float scale,
                               int iv1_begin, int iv1_end, int iv0_first, int iv0_step, void* stream);

/* MLEM/OSEM forward step fused with the data ratio: for the selected views
 * ratio = (P f == 0) ? 0 : meas / (P f), the rule of the reference's rdivide
 * (src/data_cube.cpp:150-155) applied to the projection without storing it.
 * ratio may alias meas only if meas is not needed afterwards. */
int petl_project_ratio_dev(const petl_geom* G, const float* f, const float* meas, float* ratio, int iv1_begin,
                           int iv1_end, int iv0_first, int iv0_step, void* stream);

/* nnz of the forward operator: the number of (ray, voxel) pairs with a
 * nonzero footprint weight, counted on the device; *nnz_host receives it
 * (synchronizes the stream). */
int petl_project_nnz_dev(const petl_geom* G, double* nnz_host, void* stream);

/* PFDR rebinning (src/pfdr.cu:159-315): g [N_v1][N_v0][N_u1][N_u0] ->
 * g_reb [N_v0][N_u1][N_u0]. */
int petl_pfdr_dev(const petl_geom* G, const float* g, float* g_reb, void* stream);

/* rampFilter1D (src/ramp_filter.cu:156-333) on every u0 row of a rebinned
 * planogram, in place, followed (if apply_weight) by the inverse planogram
 * weight sqrt(1+v1^2+v0^2) of apply_planogram_weight(true)
 * (src/planogram.cpp:304-333) with v1 = v1_0 of G. */
int petl_ramp_dev(const petl_geom* G, float* g_reb, int apply_weight, void* stream);

/* FBP (PETL::doFBP, src/petl.cpp:310-355) of one planogram into f:
 * f = accumulate ? f + fbp : fbp.  Needs N_v1 > 1 data (PFDR first) or an
 * already rebinned planogram when G->N_v1 == 1. */
int petl_fbp_dev(const petl_geom* G, const float* g, float* f, int accumulate, void* stream);

/* --- BF16 storage ---------------------------------------------------------
 * No reference counterpart (the reference stores float32 only).  Volumes and
 * planograms in bfloat16 (void* = __nv_bfloat16*), footprints accumulated in
 * FP32, results rounded to bfloat16 once.  These run the TMA-staged
 * shear-warp kernels only: axis-aligned planograms with bin pitch equal to
 * the voxel pitch, 16-byte aligned buffers, volume and planogram rows that
 * are multiples of 8 elements, and N_u0, numX <= 256 for the
 * backprojection.  Anything else is refused with an error. */
int petl_project_bf16_dev(const petl_geom* G, const void* f, void* g, int iv1_begin, int iv1_end, int iv0_first,
                          int iv0_step, void* stream);
/* ratio = (P f == 0) ? 0 : meas / (P f), all three in bfloat16 */
int petl_project_ratio_bf16_dev(const petl_geom* G, const void* f, const void* meas, void* ratio, int iv1_begin,
                                int iv1_end, int iv0_first, int iv0_step, void* stream);
/* f (float32) = accumulate ? f + scale*P^T g : scale*P^T g with g in bfloat16 */
int petl_backproject_bf16_dev(const petl_geom* G, const void* g, float* f, int mode, int accumulate, float scale,
                              int iv1_begin, int iv1_end, int iv0_first, int iv0_step, void* stream);
/* y (bfloat16) = x rounded to nearest even */
int petl_to_bf16_dev(const float* x, void* y, long long n, void* stream);
/* f (bfloat16) *= d / sens with the DIV rule (d/0 -> 0) */
int petl_mlem_update_bf16_dev(void* f, const float* d, const float* sens, long long n, void* stream);

/* --- reconstruction server ------------------------------------------------
 * No single reference counterpart: the reference serves one call at a time
 * through petl_server.py (src/petl_server.py:1534-1606).  A worker thread
 * owns the device and runs OSEM requests (reference-semantics
 * backprojector, f starting at 1, sensitivity zeros -> 1) with continuous
 * batching: requests are admitted in arrival order while their device
 * footprint fits hbm_budget_bytes and fewer than max_active run; requests
 * of like geometry (and subset count) share one copy of its sensitivity
 * images and projector tables, computed once and cached within the budget
 * (idle entries evicted least recently used first); every active request
 * has its own stream with up to `depth` subset steps in flight, issued
 * oldest request first while the work in flight stays under about two
 * full-size steps, so small requests overlap with large ones and new ones
 * join while others run.  Batched launches (petl_server_set_batching, off
 * by default): when a request whose subset
 * steps are too small to fill the device (under two waves of CTAs) issues a
 * step with none in flight, up to seven younger requests of its geometry
 * and subset count with no step in flight join it (each at its own
 * subset), and one launch of each split projector kernel and of the image
 * update serves them all.  Data
 * and images stay resident until the result is copied out.  A request's
 * result does not depend on what else runs, batched or not. */
void* petl_server_create(double hbm_budget_bytes, int max_active, int depth, int device);
/* g_host: the request's planogram, which must stay valid until
 * petl_server_wait returns for it; *id_out receives the request id. */
int petl_server_submit(void* server, const petl_geom* G, const float* g_host, int num_subsets, int num_iter,
                       long long* id_out);
/* The same with a deadline, deadline_s seconds after submission (< 0: none).
 * A request still pending at its deadline fails without being admitted; an
 * active one issues no further steps, lets its steps in flight finish,
 * releases its memory and fails.  Its waiter gets a nonzero return and
 * "deadline exceeded" in petl_last_error(). */
int petl_server_submit_deadline(void* server, const petl_geom* G, const float* g_host, int num_subsets, int num_iter,
                                double deadline_s, long long* id_out);
/* Cancels a request that has not been waited for: it ends as a deadline
 * does, with "cancelled".  A request that already finished is unaffected. */
int petl_server_cancel(void* server, long long id);
/* Blocks until the request finishes; copies the image (numZ*numY*numX
 * floats) to f_host when non-null; latency = submit to result on the host,
 * queue = submit to admission, both in seconds. */
int petl_server_wait(void* server, long long id, float* f_host, double* latency_s, double* queue_s);
/* out[0..5]: completed, failed, active, pending, HBM bytes reserved now,
 * peak HBM bytes reserved */
int petl_server_stats(void* server, double* out);
/* Members of a batched step at most, 1 (no batched launches, the default)
 * to 8. */
int petl_server_set_batching(void* server, int max_members);
/* out[0]: batched steps issued (two or more members), out[1]: member steps
 * they served */
int petl_server_batch_stats(void* server, double* out);
void petl_server_destroy(void* server);

/* --- regularizers, volume [N1][N2][N3] ------------------------------------ */
/* aTV_RelativeDifferencesLoss_gradient (src/relative_differences.cu:481-532) */
int petl_rd_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, void* stream);
/* Relative-difference penalty value, summed as the reference cost kernel does
 * (each pair from both sides) with the neighbour index taken correctly; *out
 * is a DEVICE double. */
int petl_rd_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, double* out, void* stream);
/* anisotropicTotalVariation_gradient / _cost / _quadraticForm
 * (src/total_variation.cu:588-811), p-Huber, 6 or 26 neighbours. cost and
 * quadform write a DEVICE double. */
int petl_tv_gradient_dev(const float* f, float* Df, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, void* stream);
int petl_tv_cost_dev(const float* f, int N1, int N2, int N3, float delta, float beta, float p, int numNeighbors,
                     double* out, void* stream);
int petl_tv_quadform_dev(const float* f, const float* d, int N1, int N2, int N3, float delta, float beta, float p,
                         int numNeighbors, double* out, void* stream);

/* gaussian_filter (src/relative_differences.cu:314-411, 753-800): in place,
 * numDims 1 filters along N1, 2 along (N2, N3), 3 along all axes. */
int petl_gaussian_filter_dev(float* f, int N1, int N2, int N3, float FWHM, int numDims, void* stream);

/* --- elementwise / reductions (dataCube rules, src/data_cube.cpp:97-166) --- */
/* denom = num/denom, 0 where denom == 0 (RDIV) */
int petl_rdivide_dev(const float* num, float* denom, long long n, void* stream);
/* x = x/y, 0 where y == 0 (DIV) */
int petl_divide_dev(float* x, const float* y, long long n, void* stream);
int petl_multiply_dev(float* x, const float* y, long long n, void* stream);
/* x = (x == 0) ? v : 1/x */
int petl_reciprocal_dev(float* x, long long n, float divide_by_zero_value, void* stream);
/* *out (device double) = sum x*y*(w ? w : 1), FP64 accumulation */
int petl_dot_dev(const float* x, const float* y, const float* w, long long n, double* out, void* stream);
/* *out (device double) = sum over Pf>0 of g*log(Pf) - Pf (Poisson log-likelihood) */
int petl_loglik_dev(const float* g, const float* Pf, long long n, double* out, void* stream);
/* Pf = (Pf > 0) ? 1 - g/Pf : 0, in place: the gradient of the Poisson
 * negative log-likelihood sum(Pf - g log Pf) (over Pf > 0) with respect to
 * Pf.  No reference counterpart (the reference has no gradient-based
 * likelihood path); used by the autograd wrappers. */
int petl_poisson_grad_dev(float* Pf, const float* g, long long n, void* stream);
/* x = a*x + b*y */
int petl_axpby_dev(float* x, const float* y, float a, float b, long long n, void* stream);
/* MLEM image update f *= d / sens with the DIV rule (d/0 -> 0) */
int petl_mlem_update_dev(float* f, const float* d, const float* sens, long long n, void* stream);
/* one-step-late RD update (src/petl_server.py:1597-1602):
 * den = max(0.1*sens, sens + Df); f *= (den == 0 ? 0 : d/den) */
int petl_osl_update_dev(float* f, const float* d, const float* sens, const float* Df, long long n, void* stream);

#ifdef __cplusplus
}
#endif
#endif
