/*
 * CPU oracle for the planogram reconstruction path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C++ (templated on float/double, OpenMP
 * over independent outputs), the arithmetic of the reference PETL kernels:
 * geometry (src/planogram.cpp), the separable-footprint projector and
 * backprojector (src/projectors.cu), PFDR (src/pfdr.cu), the ramp filter
 * (src/ramp_filter.cu), the relative-difference and Huber-TV regularizers
 * (src/relative_differences.cu, src/total_variation.cu) and the FFT size
 * helper (src/vector_ops.cpp).  Only the test-suite, the smoke check and the
 * CPU-baseline leg of the benchmark load it, always as the checker; the
 * product library never links or calls it.
 *
 * Parity of this oracle is pinned against golden vectors produced by the
 * reference library itself (tests/golden, generating script beside them).
 */
#ifndef PETL_ORACLE_H
#define PETL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One planogram plus the volume, in the units the reference stores
 * internally: psi in radians, R/L/H are HALF lengths (src/planogram.h:41-51),
 * start values are the coordinates of sample 0.  All floats, exactly as the
 * reference keeps them, so the FP64 oracle starts from identical inputs. */
typedef struct {
    float psi, R, L, H, v_m0, v_m1;
    int   N_v1, N_v0, N_u1, N_u0;
    float T_v1, T_v0, T_u1, T_u0;
    float v1_0, v0_0, u1_0, u0_0;
    float cos_psi, sin_psi;          /* float(cos(psi)), float(sin(psi)) */
    int   numX, numY, numZ;
    float voxelWidth, voxelHeight;
    float x_0, y_0, z_0;             /* parameters::x_0() etc. */
} oracle_geom;

/* planogram::init (src/planogram.cpp:143-186) + parameters::x_0/y_0/z_0
 * (src/parameters.cpp:271-284).  Arguments follow PETL::add_planogram, i.e.
 * already halved lengths and psi in radians.  Returns 0 on invalid input. */
int oracle_planogram_init(oracle_geom* G, float psi, float R, float L, float H,
                          float v_m0, float v_m1, float T);
void oracle_set_volume(oracle_geom* G, int numX, int numY, int numZ,
                       float voxelWidth, float voxelHeight,
                       float offsetX, float offsetY, float offsetZ);

/* List-mode binning of coincidences (blue[i], pink[i], xyz in mm) into one
 * planogram, in event order (src/planogram.cpp:113-141, src/binning.cpp:
 * 614-790): nearest bin (linear == 0) or bilinear deposit in (u1, u0);
 * chest_wall != 0 shifts u1 by -H.  Accumulates into g (zero it first). */
void oracle_bin_events(const oracle_geom* G, const float* blue, const float* pink, long long n, float* g,
                       int linear, int chest_wall);

/* src/vector_ops.cpp:481-505 */
int oracle_optimal_fft_size(int N);

/* Forward SF projection of one planogram (src/projectors.cu:11-238), all v1
 * slices.  f[z][y][x] -> g[v1][v0][u1][u0].  Overwrites g. */
void oracle_project_f64(const oracle_geom* G, const double* f, double* g, int nthreads);
void oracle_project_f32(const oracle_geom* G, const float* f, float* g, int nthreads);

/* Backprojection of one planogram (src/projectors.cu:240-377) summed over all
 * v1 slices, with the 2x2 texture taps replaced by exact bilinear weights
 * (texmode 0) or by an emulation of hardware linear filtering whose weights
 * carry 8 fractional bits (texmode 1: round to nearest, 2: truncate).
 * g -> f (overwrites f). */
void oracle_backproject_f64(const oracle_geom* G, const double* g, double* f, int texmode, int nthreads);
/* the views iv0 = first + k*step only (ordered subsets); exact weights */
void oracle_project_sub_f64(const oracle_geom* G, const double* f, double* g, int first, int step, int nthreads);
void oracle_backproject_sub_f64(const oracle_geom* G, const double* g, double* f, int first, int step, int nthreads);
void oracle_backproject_f32(const oracle_geom* G, const float* g, float* f, int texmode, int nthreads);

/* Count of (ray, voxel) pairs with a nonzero footprint weight in the forward
 * projector, i.e. nnz(A) for this geometry (the FLOP basis of the roofline). */
double oracle_project_nnz(const oracle_geom* G, int nthreads);
/* the same count with the footprint arithmetic in float (single != 0) */
double oracle_project_nnz_t(const oracle_geom* G, int nthreads, int single);

/* PFDR (src/pfdr.cu:59-315): g[v1][v0][u1][u0] -> g_reb[v0][u1][u0], 2-D
 * transforms done with a mixed radix double FFT. */
void oracle_pfdr_f64(const oracle_geom* G, const double* g, double* g_reb, int nthreads);

/* rampFilter1D (src/ramp_filter.cu:156-348) on rows of length N_u0;
 * nrows = N_v0 * N_u1 rows, filtered in place. */
void oracle_ramp_f64(const oracle_geom* G, double* rows, long nrows, int nthreads);

/* Complex FFT (mixed radix 2/3/other) used by the oracle; exported so that the
 * tests can pin it against numpy.  data is interleaved re/im, sign -1 forward. */
void oracle_fft_c2c(double* data, int n, int sign);

/* Relative-difference penalty gradient (src/relative_differences.cu:13-28,
 * 107-173), input clipped f<1e-8 -> 0 first.  Volume [N1][N2][N3]. */
void oracle_rd_gradient_f64(const double* f, double* Df, int N1, int N2, int N3,
                            double delta, double beta, int nthreads);
/* RD cost as the reference's cost kernel sums it, but with the corrected
 * neighbour index (the reference has an indexing slip at
 * src/relative_differences.cu:77); used for finite-difference checks. */
double oracle_rd_cost_f64(const double* f, int N1, int N2, int N3, double delta, double beta);

/* Huber-TV with USE_P_HUBER (src/total_variation.cu:21-78,80-572,574-811).
 * numNeighbors 6 or 26.  beta<=0 -> 1, delta<1e-8 -> 1e-8 as the reference. */
double oracle_tv_cost_f64(const double* f, int N1, int N2, int N3, double delta, double beta,
                          double p, int numNeighbors);
void   oracle_tv_gradient_f64(const double* f, double* Df, int N1, int N2, int N3, double delta,
                              double beta, double p, int numNeighbors, int nthreads);
double oracle_tv_quadform_f64(const double* f, const double* d, int N1, int N2, int N3,
                              double delta, double beta, double p, int numNeighbors);

/* Solid-angle factor of projection (iv1, iv0) and its application to one
 * planogram (src/planogram.cpp:262-302); inverse != 0 gives the model. */
float oracle_solid_angle_factor(const oracle_geom* G, int iv1, int iv0, int inverse);
void  oracle_solid_angle(const oracle_geom* G, float* g, int inverse);

/* src/vector_ops.cpp:358-374 */
float oracle_median(const float* x, long long n);

/* PETL::apply_corrections on one planogram: g /= r, then the bad-pixel
 * median in-fill (src/petl.cpp:163-192, src/median_filter.cu:11-190). */
void oracle_apply_corrections(const oracle_geom* G, float* g, const float* r, float rel, int nthreads);

/* An analytic solid (src/phantom.h:23-57): type 0 ellipsoid, 1
 * parallelepiped, 2-4 cylinder x/y/z, 5-7 cone x/y/z. */
typedef struct oracle_solid {
    int type;
    float centers[3], radii[3];
    float val;
    float A[9];
    float clip[6][4];
    int rotated, num_clip;
    float clip_cone[2];
    float given_c[3], given_r[3];
} oracle_solid;

/* geometricObject::init (src/phantom.cpp:535-640); 0 on invalid input. */
int oracle_solid_init(oracle_solid* s, int type, const float* c, const float* r, float val, const float* A,
                      const float* clip);
/* phantom::voxelize (src/phantom.cpp:105-335), into f [z][y][x]. */
void oracle_voxelize(const oracle_solid* s, int n, float* f, int numX, int numY, int numZ, float T_x, float T_z,
                     float x_0, float y_0, float z_0, int oversampling);
/* rayTracingKernel / stoppingPowerKernel of one planogram
 * (src/analytic_ray_tracing_gpu.cu:693-846). */
void oracle_ray_trace(const oracle_geom* G, const oracle_solid* s, int n, float* g, int oversampling, int stopping,
                      int nthreads);

#ifdef __cplusplus
}
#endif
#endif
