/*
 * petl.h -- the reference-compatible C ABI of libpetl.so (B200 build).
 *
 * Every function below replaces the function of the same name declared in the
 * reference's src/petl_c_interface.h (line given per entry); argument order,
 * units and return conventions are the same, so the reference Python binding
 * (src/petl_server.py) loads this library unchanged.  All pointers are HOST
 * pointers owned by the caller (numpy arrays in the reference binding); the
 * library copies them to the GPU, computes there and copies results back.
 * Planograms are float32 [N_v1][N_v0][N_u1][N_u0]; volumes float32
 * [numZ][numY][numX]; float** arguments hold one planogram per entry.
 *
 * Units: psi in degrees, D/L/H full lengths in mm (halved internally, as the
 * reference does at src/petl_c_interface.cpp:216-219).
 *
 * Error behaviour: bool functions return false (and print a reason to stderr)
 * on invalid input or device failure, the contract the reference binding
 * relies on (it raises on false).  Setters keep the reference's rules, e.g.
 * an offset must be positive to be accepted (src/petl_c_interface.cpp:
 * 154-200).  Every function of the reference interface computes what the
 * reference's does, on the GPU; the scatter simulation, which computes
 * nothing in the reference, validates its inputs as the reference's does.
 *
 * Device-pointer entry points for the resident path live in petl_device.h.
 */
#ifndef PETL_B200_PETL_H
#define PETL_B200_PETL_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* --- model registry (src/petl_c_interface.h:14-18) ------------------------ */
bool set_model(int i);                                   /* :14 */
int  create_new_model(void);                             /* :15 */
void about(void);                                        /* :16 */
bool copy_parameters(int param_id);                      /* :18 */
void clearAll(void);                                     /* :20 */
void print_parameters(void);                             /* :22 */
bool volume_defined(void);                               /* :23 */
bool geometry_defined(void);                             /* :24 */

/* --- volume getters / setters (src/petl_c_interface.h:26-43) --------------- */
int   get_numX(void);            bool set_numX(int);     /* :26-27 */
int   get_numY(void);            bool set_numY(int);     /* :28-29 */
int   get_numZ(void);            bool set_numZ(int);     /* :30-31 */
float get_voxelWidth(void);      bool set_voxelWidth(float);   /* :33-34 */
float get_voxelHeight(void);     bool set_voxelHeight(float);  /* :35-36 */
float get_offsetX(void);         bool set_offsetX(float);      /* :38-39 */
float get_offsetY(void);         bool set_offsetY(float);      /* :40-41 */
float get_offsetZ(void);         bool set_offsetZ(float);      /* :42-43 */

/* --- planogram geometry (src/petl_c_interface.h:45-53) --------------------- */
int  get_numPlanograms(void);                            /* :45 */
bool get_planogramSize(int which, int* shape);           /* :46  shape[4] = N_v1,N_v0,N_u1,N_u0 */
bool add_planogram(float psi, float R, float L, float H, float v_m0, float v_m1, float T); /* :48 */
bool remove_planogram(int which);                        /* :49 */
bool keep_only_planogram(int which);                     /* :50 */
bool set_default_volume(float scale);                    /* :52 */
bool set_volume(int numX, int numY, int numZ, float voxelWidth, float voxelHeight,
                float offsetX, float offsetY, float offsetZ);   /* :53 */

/* --- list-mode binning, phantoms, detector modules, scatter ---------------- */
/* List-mode binning of a coincidence file (.lst records, else the binary
 * acquisition format) into every planogram, overwriting g: bilinear in
 * (u1, u0), z from the chest wall, mm -- the reference's defaults
 * (src/petl.cpp:65-79, src/binning.cpp:558-790).  Parsed on the host in
 * batches, binned on the GPU. */
bool bin(float** g, char* file_name);                    /* :55 */
/* Scatter simulation: as the reference's, true for valid inputs and a
 * defined model, and g is left as it is (src/petl.cpp:194-202). */
bool simulate_scatter(float** g, float* mu);             /* :57 */
/* Analytic solids (type 0 ellipsoid, 1 parallelepiped, 2-4 cylinder x/y/z,
 * 5-7 cone x/y/z; A a 3x3 rotation or null; clip per axis or null) appended
 * to the model's phantom or to its detector-module model
 * (src/phantom.cpp:79-93, 535-640). */
bool add_object(int type, float* c, float* r, float val, float* A, float* clip); /* :64 */
bool add_module(int type, float* c, float* r, float val, float* A, float* clip); /* :65 */
bool clear_phantom(void);                                /* :66 */
bool clear_modules(void);                                /* :67 */
bool scale_phantom(float, float, float);                 /* :68 src/phantom.cpp:1120-1141 */
/* The phantom's solids written into f in order (values outside every solid
 * kept), 1..5 sub-samples per axis (src/phantom.cpp:105-335); on the GPU. */
bool voxelize(float* f, int oversampling);               /* :69 */
/* Analytic line integrals of every planogram through the phantom, and the
 * detector stopping power through the module model (1 everywhere without
 * modules); oversampling odd 1..11 lines per bin and axis
 * (src/analytic_ray_tracing_gpu.cu:693-994); on the GPU. */
bool ray_trace(float** g, int oversampling);             /* :70 */
bool stopping_power(float** g, int oversampling);        /* :71 */

/* --- corrections: implemented (on the GPU, host arrays in and out) --------- */
/* Every planogram's projection (iv1, iv0) times 2 pi (1 + v0^2 + v1^2)^1.5 /
 * (T_v1 T_v0), or its inverse (the solid-angle model) for do_inverse
 * (src/petl.cpp:154-162, src/planogram.cpp:262-302). */
bool set_solid_angle_correction(float** g, bool do_inverse); /* :72 */
/* g = g / r, then the bad-pixel median in-fill below threshold * median(r)
 * per projection, zero outside the field of view (src/petl.cpp:163-192,
 * src/median_filter.cu). */
bool apply_corrections(float** g, float** r, float threshold); /* :73 */

/* --- projectors and analytic reconstruction (src/petl_c_interface.h:59-62) -- */
bool project(float** g, float* f);                       /* :59  g = P f (overwrites g) */
bool backproject(float** g, float* f);                   /* :60  f = P^T g summed over planograms (overwrites f) */
bool FBP(float** g, float* f);                           /* :61  PFDR if N_v1>1, ramp, weight, backproject */
bool PFDR(float** g, float** g_reb);                     /* :62  sets N_v1=1, v1_0=0 in the model, as the reference */

/* --- elementwise / reductions (src/petl_c_interface.h:75-88) --------------- */
bool multiply3D(float* x, float* y, int N_1, int N_2, int N_3);            /* :75 x *= y */
bool multiply4D(float* x, float* y, int N_1, int N_2, int N_3, int N_4);   /* :76 */
bool divide3D(float* x, float* y, int N_1, int N_2, int N_3);              /* :78 x /= y, x/0 -> 0 */
bool divide4D(float* x, float* y, int N_1, int N_2, int N_3, int N_4);     /* :79 */
bool rdivide3D(float* num, float* denom, int N_1, int N_2, int N_3);       /* :81 denom = num/denom, denom==0 -> 0 */
bool rdivide4D(float* num, float* denom, int N_1, int N_2, int N_3, int N_4); /* :82 */
bool reciprocal3D(float* x, int N_1, int N_2, int N_3, float divide_by_zero_value);          /* :84 */
bool reciprocal4D(float* x, int N_1, int N_2, int N_3, int N_4, float divide_by_zero_value); /* :85 */
float inner_product3D(float* x, float* y, float* w, int N_1, int N_2, int N_3);              /* :87 */
float inner_product4D(float* x, float* y, float* w, int N_1, int N_2, int N_3, int N_4);     /* :88 */

/* --- regularizers (src/petl_c_interface.h:91-97) ---------------------------
 * data_on_cpu == false means f/Df/d are DEVICE pointers (the reference's
 * torch path); true means host pointers. */
float TV_cost(float* f, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu);          /* :91 */
bool  TV_gradient(float* f, float* Df, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu); /* :92 */
float TV_quadForm(float* f, float* d, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu);  /* :93 */
bool  diffuse(float* f, int N_1, int N_2, int N_3, float delta, float p, int numIter, bool data_on_cpu);         /* :94 */
bool  TV_denoise(float* f, int N_1, int N_2, int N_3, float delta, float beta, float p, int numIter, bool doMean, bool data_on_cpu); /* :95 */
bool  relativeDifferences_gradient(float* f, float* Df, int N_1, int N_2, int N_3, float delta, float beta);  /* :96 */
bool  gaussian_filter(float* f, int N_1, int N_2, int N_3, float FWHM, int numDims);                          /* :97 */

#ifdef __cplusplus
}
#endif
#endif
