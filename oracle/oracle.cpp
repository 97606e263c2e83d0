// CPU oracle for the planogram reconstruction path -- TEST INFRASTRUCTURE ONLY.
//
// A restatement of the reference PETL algorithms in portable C++ (templated on
// the arithmetic type, OpenMP over independent outputs).  It is the checker of
// the CUDA library and the CPU baseline of the benchmark; the product never
// links it.  Every routine cites the reference file:line it follows (paths are
// relative to the reference project root).  Its agreement with the reference
// itself is pinned by golden vectors produced from the reference library
// (tests/golden).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

const double kPI = 3.141592653589793;  // src/petl_defines.h

template <class T> inline T tabs(T x) { return x < T(0) ? -x : x; }
template <class T> inline T tmin(T a, T b) { return a < b ? a : b; }
template <class T> inline T tmax(T a, T b) { return a > b ? a : b; }

inline void set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}

// The forward projector's ray masks (src/projectors.cu:19-43) in float with
// fused multiply-adds, as nvcc compiles them: v = fma(i, T, start),
// |u| - T/2 > L + R|v0|  and  |u1| - T/2 > H - R|v1|.
inline bool ray_visible(const oracle_geom& G, int iv1, int iv0, int iu1, int iu0)
{
    const float v1 = std::fma(float(iv1), G.T_v1, G.v1_0);
    const float v0 = std::fma(float(iv0), G.T_v0, G.v0_0);
    const float u1 = std::fma(float(iu1), G.T_u1, G.u1_0);
    const float u0 = std::fma(float(iu0), G.T_u0, G.u0_0);
    if (std::fabs(u0) - 0.5f * G.T_u0 > std::fma(G.R, std::fabs(v0), G.L)) return false;
    if (std::fabs(u1) - 0.5f * G.T_u1 > std::fma(-G.R, std::fabs(v1), G.H)) return false;
    return true;
}

// The reference backprojector's voxel visibility test (src/projectors.cu:289)
// in float: u1 = fma(v1, t, z) with v1 = fma(iv1, T_v1, v1_0).
inline bool voxel_visible(const oracle_geom& G, int iv1, float z, float t)
{
    const float v1 = std::fma(float(iv1), G.T_v1, G.v1_0);
    const float u1 = std::fma(v1, t, z);
    return std::fabs(u1) - 0.5f * G.T_u1 <= std::fma(-G.R, std::fabs(v1), G.H);
}

// ---------------------------------------------------------------------------
// Forward projector: src/projectors.cu:11-238 (one ray per (iv1,iv0,iu1,iu0)).
// Texture reads at voxel centres are exact; out-of-volume voxels are never
// touched because the index ranges are clamped (lines 95-101, 150-156).
// ---------------------------------------------------------------------------
template <class T>
T project_ray(const oracle_geom& G, const T* f, int iv1, int iv0, int iu1, int iu0, double* nnz)
{
    const T cos_psi = T(G.cos_psi), sin_psi = T(G.sin_psi);
    const T R = T(G.R), L = T(G.L), H = T(G.H);
    const T Tg_w = T(G.T_v1), Tg_x = T(G.T_v0), Tg_y = T(G.T_u1), Tg_z = T(G.T_u0);
    const T sg_w = T(G.v1_0), sg_x = T(G.v0_0), sg_y = T(G.u1_0), sg_z = T(G.u0_0);
    const T Tf_x = T(G.voxelWidth), Tf_y = T(G.voxelWidth), Tf_z = T(G.voxelHeight);
    const T sf_x = T(G.x_0), sf_y = T(G.y_0), sf_z = T(G.z_0);
    const int Nx = G.numX, Ny = G.numY, Nz = G.numZ;

    const T v1 = T(iv1) * Tg_w + sg_w;
    const T v0 = T(iv0) * Tg_x + sg_x;
    const T u1 = T(iu1) * Tg_y + sg_y;
    const T u0 = T(iu0) * Tg_z + sg_z;

    // early exits, lines 30-43.  These are yes/no decisions that sit exactly
    // on ties for some geometries, so they are taken in float the way the
    // reference's compiled kernel takes them (a*b+c contracted into one fma).
    (void)L; (void)H; (void)R;
    if (!ray_visible(G, iv1, iv0, iu1, iu0)) return T(0);

    const T iu0_min = T(iu0) - T(0.5), iu0_max = T(iu0) + T(0.5);
    const T iu1_min = T(iu1) - T(0.5), iu1_max = T(iu1) + T(0.5);

    const T p_x = u0 * cos_psi, p_y = u0 * sin_psi, p_z = u1;
    const T r_x = -(v0 * cos_psi + sin_psi), r_y = -(v0 * sin_psi - cos_psi), r_z = -v1;

    const T Tx_inv = T(1) / Tf_x, Ty_inv = T(1) / Tf_y, Tz_inv = T(1) / Tf_z;
    const T Tu1_inv = T(1) / Tg_y, Tu0_inv = T(1) / Tg_z;
    const T width_z = T(0.5) * Tg_y;
    const T Tz_over_Tu1 = Tf_z * Tu1_inv;
    const T z_fw = T(0.5) * Tf_z * Tu1_inv;

    T val = T(0);
    double count = 0.0;
    const T* fz;
    // the driving axis is a yes/no decision that sits exactly on a tie for
    // some views (|r_x| = |r_y|: psi = 135 degrees at v0 = 0), so it is taken
    // in float with the contracted fma of the reference's compiled kernel,
    // as the ray masks are (lines 62-65)
    const float v0f = std::fma(float(iv0), G.T_v0, G.v0_0);
    const float rxf = -std::fma(v0f, G.cos_psi, G.sin_psi), ryf = -std::fma(v0f, G.sin_psi, -G.cos_psi);
    if (std::fabs(rxf) >= std::fabs(ryf)) {
        // x-driven branch, lines 77-130
        const T width_y = T(0.5) * Tg_z * tabs(sin_psi);
        const T sin_psi_inv = T(1) / sin_psi;
        const T rx_inv = T(1) / r_x;
        const T l_phi = Tf_x * tabs(sin_psi_inv);
        const T y_fw = T(0.5) * Tf_y * tabs(sin_psi_inv) * Tu0_inv;
        for (int ix = 0; ix < Nx; ix++) {
            const T x = T(ix) * Tf_x + sf_x;
            const T t = (x - p_x) * rx_inv;
            const T y_c = p_y + t * r_y, z_c = p_z + t * r_z;
            const T y_A = y_c - width_y, y_B = y_c + width_y;
            const int iy_min = std::max(0, int(std::ceil((y_A - T(0.5) * Tf_y - sf_y) * Ty_inv)));
            const int iy_max = std::min(Ny - 1, int(std::floor((y_B + T(0.5) * Tf_y - sf_y) * Ty_inv)));
            const T z_A = z_c - width_z, z_B = z_c + width_z;
            const int iz_min = std::max(0, int(std::ceil((z_A - T(0.5) * Tf_z - sf_z) * Tz_inv)));
            const int iz_max = std::min(Nz - 1, int(std::floor((z_B + T(0.5) * Tf_z - sf_z) * Tz_inv)));
            T y = T(iy_min) * Tf_y + sf_y - t * r_y;
            const T z_start = (T(iz_min) * Tf_z + sf_z - t * r_z - sg_y) * Tu1_inv;
            for (int iy = iy_min; iy <= iy_max; iy++) {
                const T c = (y * sin_psi_inv - sg_z) * Tu0_inv;
                const T fp = tmin(iu0_max, c + y_fw) - tmax(iu0_min, c - y_fw);
                if (fp > T(0)) {
                    T z = z_start;
                    for (int iz = iz_min; iz <= iz_max; iz++) {
                        const T fz1 = tmax(T(0), tmin(iu1_max, z + z_fw) - tmax(iu1_min, z - z_fw));
                        if (fz1 > T(0)) {
                            if (f) val += f[(size_t(iz) * Ny + iy) * Nx + ix] * fp * fz1;
                            count += 1.0;
                        }
                        z += Tz_over_Tu1;
                    }
                }
                y += Tf_y;
            }
        }
        val *= l_phi;
    } else {
        // y-driven branch, lines 131-185
        const T width_x = T(0.5) * Tg_z * tabs(cos_psi);
        const T cos_psi_inv = T(1) / cos_psi;
        const T ry_inv = T(1) / r_y;
        const T l_phi = Tf_x * tabs(cos_psi_inv);
        const T x_fw = T(0.5) * Tf_x * tabs(cos_psi_inv) * Tu0_inv;
        for (int iy = 0; iy < Ny; iy++) {
            const T y = T(iy) * Tf_y + sf_y;
            const T t = (y - p_y) * ry_inv;
            const T x_c = p_x + t * r_x, z_c = p_z + t * r_z;
            const T x_A = x_c - width_x, x_B = x_c + width_x;
            const int ix_min = std::max(0, int(std::ceil((x_A - T(0.5) * Tf_x - sf_x) * Tx_inv)));
            const int ix_max = std::min(Nx - 1, int(std::floor((x_B + T(0.5) * Tf_x - sf_x) * Tx_inv)));
            const T z_A = z_c - width_z, z_B = z_c + width_z;
            const int iz_min = std::max(0, int(std::ceil((z_A - T(0.5) * Tf_z - sf_z) * Tz_inv)));
            const int iz_max = std::min(Nz - 1, int(std::floor((z_B + T(0.5) * Tf_z - sf_z) * Tz_inv)));
            T x = T(ix_min) * Tf_x + sf_x - t * r_x;
            const T z_start = (T(iz_min) * Tf_z + sf_z - t * r_z - sg_y) * Tu1_inv;
            for (int ix = ix_min; ix <= ix_max; ix++) {
                const T c = (x * cos_psi_inv - sg_z) * Tu0_inv;
                const T fp = tmin(iu0_max, c + x_fw) - tmax(iu0_min, c - x_fw);
                if (fp > T(0)) {
                    T z = z_start;
                    for (int iz = iz_min; iz <= iz_max; iz++) {
                        const T fz1 = tmax(T(0), tmin(iu1_max, z + z_fw) - tmax(iu1_min, z - z_fw));
                        if (fz1 > T(0)) {
                            if (f) val += f[(size_t(iz) * Ny + iy) * Nx + ix] * fp * fz1;
                            count += 1.0;
                        }
                        z += Tz_over_Tu1;
                    }
                }
                x += Tf_x;
            }
        }
        val *= l_phi;
    }
    (void)fz;
    if (nnz) *nnz += count;
    // line 237
    return val * (T(1) / std::sqrt(T(1) + v0 * v0 + v1 * v1));
}

// views iv0 = first, first + step, ...; the other views are set to zero
template <class T>
void project(const oracle_geom& G, const T* f, T* g, int nthreads, int first = 0, int step = 1, int v1b = 0,
             int v1e = -1)
{
    // g holds the v1 slices [v1b, v1e) only (all of them by default)
    set_threads(nthreads);
    if (v1e < 0) v1e = G.N_v1;
    const long nview = long(v1e - v1b) * G.N_v0;
#pragma omp parallel for schedule(dynamic)
    for (long v = 0; v < nview; v++) {
        const int iv1 = v1b + int(v / G.N_v0), iv0 = int(v % G.N_v0);
        T* gv = g + size_t(v) * G.N_u1 * G.N_u0;
        const bool in = iv0 >= first && (iv0 - first) % step == 0;
        for (int iu1 = 0; iu1 < G.N_u1; iu1++)
            for (int iu0 = 0; iu0 < G.N_u0; iu0++)
                gv[size_t(iu1) * G.N_u0 + iu0] = in ? project_ray<T>(G, f, iv1, iv0, iu1, iu0, nullptr) : T(0);
    }
}

// ---------------------------------------------------------------------------
// Backprojector: src/projectors.cu:240-377 and the per-v1 loop of
// backproject_SF (src/projectors.cu:480-489): f = sum_v1 (val_v1 * T_x).
// Each 2x2 texture fetch of the reference (line 368) is a bilinear read at
// iu0 + w_b/(w_a+w_b) scaled by (w_a+w_b); with exact weights this is
// w_a*g[iu0] + w_b*g[iu0+1], border texels read as zero.
// ---------------------------------------------------------------------------
template <class T>
inline T gat(const T* g, const oracle_geom& G, int iv0, int iu1, int iu0)
{
    if (iu0 < 0 || iu0 >= G.N_u0 || iu1 < 0 || iu1 >= G.N_u1) return T(0);
    return g[(size_t(iv0) * G.N_u1 + iu1) * G.N_u0 + iu0];
}

// one axis of the hardware linear filter: x is the texel-space coordinate as
// the reference passes it (index + shift + 0.5), returns base index and weight
inline void texaxis(float x, int mode, int& i, double& a)
{
    const float xb = x - 0.5f;
    const float fl = std::floor(xb);
    i = int(fl);
    double frac = double(xb - fl);
    if (mode == 1) frac = std::nearbyint(frac * 256.0) / 256.0;
    else if (mode == 2) frac = std::floor(frac * 256.0) / 256.0;
    a = frac;
}

// only the views iv0 = first, first + step, ... contribute
template <class T>
void backproject(const oracle_geom& G, const T* g, T* f, int texmode, int nthreads, int first = 0, int step = 1,
                 int v1b = 0, int v1e = -1)
{
    // g holds the v1 slices [v1b, v1e) only (all of them by default); only
    // those slices are summed
    set_threads(nthreads);
    if (v1e < 0) v1e = G.N_v1;
    const T cos_psi = T(G.cos_psi), sin_psi = T(G.sin_psi);
    const T R = T(G.R), H = T(G.H);
    const T Tg_w = T(G.T_v1), Tg_x = T(G.T_v0), Tg_y = T(G.T_u1), Tg_z = T(G.T_u0);
    const T sg_w = T(G.v1_0), sg_x = T(G.v0_0), sg_y = T(G.u1_0), sg_z = T(G.u0_0);
    const T Tf_x = T(G.voxelWidth), Tf_y = T(G.voxelWidth), Tf_z = T(G.voxelHeight);
    const T sf_x = T(G.x_0), sf_y = T(G.y_0), sf_z = T(G.z_0);
    const size_t plan_sz = size_t(G.N_v0) * G.N_u1 * G.N_u0;
    const long nrows = long(G.numZ) * G.numY;
#pragma omp parallel for schedule(dynamic)
    for (long r = 0; r < nrows; r++) {
        const int iz = int(r / G.numY), iy = int(r % G.numY);
        for (int ix = 0; ix < G.numX; ix++) {
            const T x = T(ix) * Tf_x + sf_x, y = T(iy) * Tf_y + sf_y, z = T(iz) * Tf_z + sf_z;
            T acc = T(0);
            for (int iv1 = v1b; iv1 < v1e; iv1++) {
                const T* gs = g + size_t(iv1 - v1b) * plan_sz;
                const T v1 = T(iv1) * Tg_w + sg_w;
                const T t = y * cos_psi - x * sin_psi;
                const T u1 = z + v1 * t;
                T val = T(0);
                const float xf = std::fma(float(ix), G.voxelWidth, G.x_0);
                const float yf = std::fma(float(iy), G.voxelWidth, G.y_0);
                const float zf = std::fma(float(iz), G.voxelHeight, G.z_0);
                const float tf = std::fma(yf, G.cos_psi, -(xf * G.sin_psi));
                (void)R; (void)H;
                if (voxel_visible(G, iv1, zf, tf)) {
                    const T x_dot_theta = x * cos_psi + y * sin_psi;
                    const T Tu1_inv = T(1) / Tg_y, Tu0_inv = T(1) / Tg_z;
                    const T iu1_mid = (u1 - sg_y) * Tu1_inv;
                    const T iu1_A = iu1_mid - T(0.5) * Tf_z * Tu1_inv;
                    const T iu1_B = iu1_mid + T(0.5) * Tf_z * Tu1_inv;
                    const int iu1_min = int(std::ceil(iu1_A - T(0.5)));
                    const int iu1_max = int(std::floor(iu1_B + T(0.5)));
                    const T xdt_dy = T(0.5) * Tf_y * sin_psi, t_dy = T(0.5) * Tf_y * cos_psi;
                    const T xdt_dx = T(0.5) * Tf_x * cos_psi, t_dx = -T(0.5) * Tf_x * sin_psi;
                    for (int iv0 = first; iv0 < G.N_v0; iv0 += step) {
                        const T v0 = T(iv0) * Tg_x + sg_x;
                        const T width_y = v0 * cos_psi + sin_psi;
                        const T width_x = cos_psi - v0 * sin_psi;
                        const T l_phi = T(1) / tmax(tabs(width_y), tabs(width_x)) *
                                        (T(1) / std::sqrt(T(1) + v0 * v0 + v1 * v1));
                        // which corner pair bounds the footprint is a yes/no
                        // decision with ties (|width_y| = |width_x| at psi = 135
                        // degrees, v0 = 0): taken in float with the reference
                        // kernel's contracted fmas
                        const float v0f = std::fma(float(iv0), G.T_v0, G.v0_0);
                        const float wyf = std::fma(v0f, G.cos_psi, G.sin_psi);
                        const float wxf = std::fma(-v0f, G.sin_psi, G.cos_psi);
                        T A, B;
                        if (std::fabs(wyf) > std::fabs(wxf)) {
                            const T lo = (x_dot_theta - xdt_dy + v0 * (t - t_dy) - sg_z) * Tu0_inv;
                            const T hi = (x_dot_theta + xdt_dy + v0 * (t + t_dy) - sg_z) * Tu0_inv;
                            if (wyf >= 0.0f) { A = lo; B = hi; } else { A = hi; B = lo; }
                        } else {
                            const T lo = (x_dot_theta - xdt_dx + v0 * (t - t_dx) - sg_z) * Tu0_inv;
                            const T hi = (x_dot_theta + xdt_dx + v0 * (t + t_dx) - sg_z) * Tu0_inv;
                            if (wxf >= 0.0f) { A = lo; B = hi; } else { A = hi; B = lo; }
                        }
                        const int iu0_min = int(std::ceil(A - T(0.5)));
                        const int iu0_max = int(std::floor(B + T(0.5)));
                        for (int iu0 = iu0_min; iu0 <= iu0_max; iu0 += 2) {
                            const T w0b = tmax(T(0), tmin(T(iu0 + 1) + T(0.5), B) - tmax(T(iu0 + 1) - T(0.5), A));
                            const T w0a = tmax(T(0), tmin(T(iu0) + T(0.5), B) - tmax(T(iu0) - T(0.5), A));
                            const T w0s = w0b + w0a;
                            if (!(w0s > T(0))) continue;
                            for (int iu1 = iu1_min; iu1 <= iu1_max; iu1 += 2) {
                                const T w1b = tmax(T(0), tmin(T(iu1 + 1) + T(0.5), iu1_B) - tmax(T(iu1 + 1) - T(0.5), iu1_A));
                                const T w1a = tmax(T(0), tmin(T(iu1) + T(0.5), iu1_B) - tmax(T(iu1) - T(0.5), iu1_A));
                                const T w1s = w1b + w1a;
                                if (!(w1s > T(0))) continue;
                                T sample;
                                if (texmode == 0) {
                                    sample = (w0a * w1a * gat(gs, G, iv0, iu1, iu0) +
                                              w0b * w1a * gat(gs, G, iv0, iu1, iu0 + 1) +
                                              w0a * w1b * gat(gs, G, iv0, iu1 + 1, iu0) +
                                              w0b * w1b * gat(gs, G, iv0, iu1 + 1, iu0 + 1));
                                    sample *= l_phi;
                                } else {
                                    // coordinates exactly as the reference forms them (float)
                                    const float s0 = float(w0b) / float(w0s), s1 = float(w1b) / float(w1s);
                                    const float cx = float(iu0) + s0 + 0.5f, cy = float(iu1) + s1 + 0.5f;
                                    int i0, i1; double a0, a1;
                                    texaxis(cx, texmode, i0, a0);
                                    texaxis(cy, texmode, i1, a1);
                                    const double b = (1 - a0) * (1 - a1) * double(gat(gs, G, iv0, i1, i0)) +
                                                     a0 * (1 - a1) * double(gat(gs, G, iv0, i1, i0 + 1)) +
                                                     (1 - a0) * a1 * double(gat(gs, G, iv0, i1 + 1, i0)) +
                                                     a0 * a1 * double(gat(gs, G, iv0, i1 + 1, i0 + 1));
                                    sample = T(b) * l_phi * w0s * w1s;
                                }
                                val += sample;
                            }
                        }
                    }
                }
                acc += val * Tf_x;
            }
            f[(size_t(iz) * G.numY + iy) * G.numX + ix] = acc;
        }
    }
}

// ---------------------------------------------------------------------------
// FFT helpers.  A plain recursive mixed-radix DFT in double precision.
// ---------------------------------------------------------------------------
typedef std::complex<double> cd;

void fft_rec(cd* x, int n, int sign, cd* scratch)
{
    if (n == 1) return;
    int p = 2;
    while (p * p <= n && n % p) p++;
    if (n % p) p = n;
    const int m = n / p;
    for (int r = 0; r < p; r++)
        for (int j = 0; j < m; j++) scratch[r * m + j] = x[j * p + r];
    for (int r = 0; r < p; r++) fft_rec(scratch + r * m, m, sign, x);
    std::vector<cd> out(n);
    for (int k = 0; k < n; k++) {
        cd s = 0;
        const int kk = k % m;
        for (int r = 0; r < p; r++) {
            const double ang = sign * 2.0 * kPI * double((long long)r * k % n) / n;
            s += scratch[r * m + kk] * cd(std::cos(ang), std::sin(ang));
        }
        out[k] = s;
    }
    for (int k = 0; k < n; k++) x[k] = out[k];
}

void fft(cd* x, int n, int sign)
{
    std::vector<cd> scratch(n);
    fft_rec(x, n, sign, scratch.data());
}

// R2C of a real row of length n -> n/2+1 bins
void r2c(const double* in, cd* out, int n)
{
    std::vector<cd> t(n);
    for (int i = 0; i < n; i++) t[i] = in[i];
    fft(t.data(), n, -1);
    for (int k = 0; k <= n / 2; k++) out[k] = t[k];
}

// unnormalized C2R of n/2+1 bins -> n reals; the imaginary parts of bin 0 and
// bin n/2 are ignored (the Hermitian completion of the half spectrum)
void c2r(const cd* in, double* out, int n)
{
    std::vector<cd> t(n);
    for (int k = 0; k <= n / 2; k++) t[k] = in[k];
    t[0] = cd(in[0].real(), 0);
    if (n % 2 == 0) t[n / 2] = cd(in[n / 2].real(), 0);
    for (int k = n / 2 + 1; k < n; k++) t[k] = std::conj(in[n - k]);
    fft(t.data(), n, +1);
    for (int i = 0; i < n; i++) out[i] = t[i].real();
}

// ---------------------------------------------------------------------------
// Regularizer helpers (src/relative_differences.cu:13-28,
// src/total_variation.cu:33-78 with USE_P_HUBER).
// ---------------------------------------------------------------------------
inline double rd(double x, double y, double delta)
{
    if (x == y) return 0.0;
    return (x - y) * (x - y) / ((x + y) + delta * std::fabs(x - y));
}
inline double drd(double x, double y, double delta)
{
    if (x == 0.0 && y == 0.0) return 0.0;
    const double s = x + y + delta * std::fabs(x - y);
    return (x - y) * (delta * std::fabs(x - y) + x + 3.0 * y) / (s * s);
}

struct Huber {
    double p, delta, slope, shift;
    Huber(double delta_, double p_) : p(p_), delta(delta_)
    {
        // setConstantMemoryParameters, src/total_variation.cu:574-586 (float constants)
        slope = double(float(std::pow(delta, 2.0 - p) / p));
        shift = double(float(delta * delta * (0.5 - 1.0 / p)));
    }
    double h(double x) const { return std::fabs(x) <= delta ? 0.5 * x * x : slope * std::pow(std::fabs(x), p) + shift; }
    double dh(double x) const { return std::fabs(x) <= delta ? x : p * slope * std::pow(std::fabs(x), p) / x; }
    double ddh(double x) const { return std::fabs(x) <= delta ? 1.0 : p * slope * std::pow(std::fabs(x), p - 2.0); }
};

// neighbourhood offsets of the 26-neighbour stencil grouped by distance
struct Nbr { int di, dj, dk, cls; };
std::vector<Nbr> neighbours(bool planar, int numNeighbors)
{
    std::vector<Nbr> v;
    for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
            for (int dk = -1; dk <= 1; dk++) {
                if (!di && !dj && !dk) continue;
                if (planar && di) continue;
                const int cls = std::abs(di) + std::abs(dj) + std::abs(dk);
                if (numNeighbors == 6 && cls > 1) continue;
                if (planar && numNeighbors == 6 && cls > 1) continue;
                v.push_back({di, dj, dk, cls});
            }
    return v;
}
inline double dist_w(int cls, double beta)
{
    return cls == 1 ? double(1.0f * float(beta))
         : cls == 2 ? double(0.7071067811865475f * float(beta))
                    : double(0.5773502691896258f * float(beta));
}

}  // namespace

extern "C" {

int oracle_optimal_fft_size(int N)
{
    // src/vector_ops.cpp:481-505: smallest 2^(n+1)*3^m >= N
    if (N <= 2) return 2;
    const double c1 = std::log2(double(N) / 2.0) / std::log2(3);
    const double c2 = 1.0 / std::log2(3);
    const double xbar = std::log2(double(N) / 2.0);
    int minValue = int(std::pow(2, int(std::ceil(xbar)) + 1));
    for (int x = 0; x < int(std::ceil(xbar)); x++) {
        const int y = int(std::ceil(c1 - c2 * double(x)));
        const int v = int(std::pow(2, x + 1) * std::pow(3, y));
        if (v < minValue && y >= 0) minValue = v;
    }
    return minValue;
}

int oracle_planogram_init(oracle_geom* G, float psi, float R, float L, float H, float v_m0, float v_m1, float T)
{
    // src/planogram.cpp:143-186 (float storage, mixed float/double arithmetic)
    if (R <= 0.0 || L <= 0.0 || H <= 0.0 || v_m0 <= 0.0 || v_m1 < 0.0 || T <= 0.0) return 0;
    G->psi = psi; G->R = R; G->L = L; G->H = H;
    G->v_m0 = v_m0;
    G->v_m1 = std::min(H / R, v_m1);
    G->T_u0 = T; G->T_u1 = T;
    G->T_v0 = G->T_u0 / R;
    G->T_v1 = G->T_u1 / R;
    G->N_u0 = 2 * int((L + R * v_m0) / G->T_u0);
    G->N_u1 = 2 * int(H / G->T_u1);
    G->N_v0 = 2 * int(v_m0 / G->T_v0) + 1;
    G->N_v1 = 2 * int(G->v_m1 / G->T_v1) + 1;
    G->T_v0 = float(v_m0 * 2.0 / float(G->N_v0));
    G->u0_0 = float(-G->T_u0 * float(G->N_u0 - 1) / 2.0);
    G->u1_0 = float(-G->T_u1 * float(G->N_u1 - 1) / 2.0);
    G->v0_0 = float(-G->T_v0 * float(G->N_v0 - 1) / 2.0);
    G->v1_0 = float(-G->T_v1 * float(G->N_v1 - 1) / 2.0);
    G->cos_psi = float(std::cos(double(psi)));
    G->sin_psi = float(std::sin(double(psi)));
    return 1;
}

void oracle_set_volume(oracle_geom* G, int numX, int numY, int numZ, float voxelWidth, float voxelHeight,
                       float offsetX, float offsetY, float offsetZ)
{
    // src/parameters.cpp:250-284
    G->numX = numX; G->numY = numY; G->numZ = numZ;
    G->voxelWidth = voxelWidth; G->voxelHeight = voxelHeight;
    G->x_0 = float((0.0 - 0.5 * (numX - 1)) * voxelWidth + offsetX);
    G->y_0 = float((0.0 - 0.5 * (numY - 1)) * voxelWidth + offsetY);
    G->z_0 = float((0.0 - 0.5 * (numZ - 1)) * voxelHeight + offsetZ);
}

void oracle_project_f64(const oracle_geom* G, const double* f, double* g, int n) { project<double>(*G, f, g, n); }
void oracle_project_sub_f64(const oracle_geom* G, const double* f, double* g, int first, int step, int n)
{
    project<double>(*G, f, g, n, first, step);
}
void oracle_backproject_sub_f64(const oracle_geom* G, const double* g, double* f, int first, int step, int n)
{
    backproject<double>(*G, g, f, 0, n, first, step);
}
void oracle_project_f32(const oracle_geom* G, const float* f, float* g, int n) { project<float>(*G, f, g, n); }
void oracle_project_band_f64(const oracle_geom* G, const double* f, double* g, int v1b, int v1e, int n)
{
    project<double>(*G, f, g, n, 0, 1, v1b, v1e);
}
void oracle_backproject_band_f64(const oracle_geom* G, const double* g, double* f, int v1b, int v1e, int n)
{
    backproject<double>(*G, g, f, 0, n, 0, 1, v1b, v1e);
}
void oracle_project_band_f32(const oracle_geom* G, const float* f, float* g, int v1b, int v1e, int n)
{
    project<float>(*G, f, g, n, 0, 1, v1b, v1e);
}
void oracle_backproject_band_f32(const oracle_geom* G, const float* g, float* f, int v1b, int v1e, int n)
{
    backproject<float>(*G, g, f, 0, n, 0, 1, v1b, v1e);
}
void oracle_backproject_f64(const oracle_geom* G, const double* g, double* f, int tm, int n) { backproject<double>(*G, g, f, tm, n); }
void oracle_backproject_f32(const oracle_geom* G, const float* g, float* f, int tm, int n) { backproject<float>(*G, g, f, tm, n); }

double oracle_project_nnz(const oracle_geom* G, int nthreads) { return oracle_project_nnz_t(G, nthreads, 0); }

double oracle_project_nnz_t(const oracle_geom* G, int nthreads, int single)
{
    set_threads(nthreads);
    const long nview = long(G->N_v1) * G->N_v0;
    double total = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (long v = 0; v < nview; v++) {
        const int iv1 = int(v / G->N_v0), iv0 = int(v % G->N_v0);
        double c = 0.0;
        for (int iu1 = 0; iu1 < G->N_u1; iu1++)
            for (int iu0 = 0; iu0 < G->N_u0; iu0++)
                if (single) project_ray<float>(*G, (const float*)nullptr, iv1, iv0, iu1, iu0, &c);
                else project_ray<double>(*G, (const double*)nullptr, iv1, iv0, iu1, iu0, &c);
        total += c;
    }
    return total;
}

void oracle_fft_c2c(double* data, int n, int sign) { fft(reinterpret_cast<cd*>(data), n, sign); }

void oracle_pfdr_f64(const oracle_geom* G, const double* g, double* g_reb, int nthreads)
{
    // src/pfdr.cu:159-315 with the kernels at 43-157.
    set_threads(nthreads);
    const int NX = oracle_optimal_fft_size(G->N_u0), NXH = NX / 2 + 1;
    const int NY = oracle_optimal_fft_size(G->N_v0);
    const int B = G->N_u1;
    const float T_U = float(1.0 / (NX * G->T_u0));
    const float T_V = float(1.0 / (NY * G->T_v0));
    const float aperture = float(1 / (2.0 * G->T_u1 * 2.0 * G->v_m0));
    (void)T_V;
    std::vector<cd> Greb(size_t(B) * NY * NXH, cd(0, 0));
    std::vector<double> W(size_t(B) * NY * NXH, 0.0);
    const size_t plan_sz = size_t(G->N_v0) * G->N_u1 * G->N_u0;
    for (int iv1 = 0; iv1 < G->N_v1; iv1++) {
        const float v1 = float(iv1) * G->T_v1 + G->v1_0;  // planogram::v1
        const double* gs = g + size_t(iv1) * plan_sz;
#pragma omp parallel for schedule(dynamic)
        for (int iu1 = 0; iu1 < B; iu1++) {
            // copy_data_to_2d_fft_buffer, weighted by 1/sqrt(1+v1^2+v0^2)
            std::vector<cd> buf(size_t(NY) * NX, cd(0, 0));
            for (int iv0 = 0; iv0 < G->N_v0; iv0++) {
                const double v0 = double(float(G->T_v0 * float(iv0) + G->v0_0));
                const double w = 1.0 / std::sqrt(1.0 + double(v1) * v1 + v0 * v0);
                for (int iu0 = 0; iu0 < G->N_u0; iu0++)
                    buf[size_t(iv0) * NX + iu0] = gs[(size_t(iv0) * G->N_u1 + iu1) * G->N_u0 + iu0] * w;
            }
            // 2-D forward transform: rows (NX) then columns (NY)
            for (int r = 0; r < NY; r++) fft(&buf[size_t(r) * NX], NX, -1);
            std::vector<cd> col(NY);
            for (int k = 0; k < NXH; k++) {
                for (int r = 0; r < NY; r++) col[r] = buf[size_t(r) * NX + k];
                fft(col.data(), NY, -1);
                for (int r = 0; r < NY; r++) buf[size_t(r) * NX + k] = col[r];
            }
            // rebin (src/pfdr.cu:78-124); the oblique u1 index is taken from u1
            // itself (line 107), so the accumulation stays in row iu1 unless
            // rounding moves it to a neighbour row
            const float u1 = float(iu1) * G->T_u1 + G->u1_0;
            const float abs_v1 = std::fabs(v1);
            for (int iV0 = 0; iV0 < NY; iV0++)
                for (int iU0 = 0; iU0 < NXH; iU0++) {
                    const float U_0 = iU0 < NX / 2 ? float(iU0) * T_U : float(iU0 - NX) * T_U;
                    if (!(abs_v1 <= 0.5f * G->T_v1 || std::fabs(U_0) > abs_v1 * aperture)) continue;
                    const size_t o = (size_t(iu1) * NY + iV0) * NXH + iU0;
                    if (abs_v1 <= 0.5f * G->T_v1) {
                        Greb[o] += buf[size_t(iV0) * NX + iU0];
                        W[o] += 1.0;
                    } else {
                        // iu1_oblique = (u1 - u1_0)/T_u1 equals iu1 (exactly so
                        // for pitches that are powers of two), hence lo = iu1,
                        // d = 0 and the sample lands in its own row
                        const float iu1_ob = (u1 - G->u1_0) / G->T_u1;
                        if (iu1_ob >= 0.0f && iu1_ob <= float(G->N_u1 - 1)) {
                            Greb[o] += buf[size_t(iV0) * NX + iU0];
                            W[o] += 1.0;
                        }
                    }
                }
        }
    }
    // normalize (src/pfdr.cu:126-142), C2R per u1 row, crop, * sqrt(1+v0^2)
#pragma omp parallel for schedule(dynamic)
    for (int iu1 = 0; iu1 < B; iu1++) {
        std::vector<cd> spec(size_t(NY) * NXH);
        for (int iV0 = 0; iV0 < NY; iV0++)
            for (int iU0 = 0; iU0 < NXH; iU0++) {
                const size_t o = (size_t(iu1) * NY + iV0) * NXH + iU0;
                double w = 1.0 / double(NY * NX);
                if (W[o] > 0.0 && iU0 != 0) w *= 1.0 / W[o];
                spec[size_t(iV0) * NXH + iU0] = Greb[o] * w;
            }
        // inverse along columns (NY), then C2R along rows (NX)
        std::vector<cd> col(NY);
        for (int k = 0; k < NXH; k++) {
            for (int r = 0; r < NY; r++) col[r] = spec[size_t(r) * NXH + k];
            fft(col.data(), NY, +1);
            for (int r = 0; r < NY; r++) spec[size_t(r) * NXH + k] = col[r];
        }
        std::vector<double> row(NX);
        for (int iv0 = 0; iv0 < G->N_v0; iv0++) {
            c2r(&spec[size_t(iv0) * NXH], row.data(), NX);
            const double v0 = double(float(G->T_v0 * float(iv0) + G->v0_0));
            const double s = std::sqrt(1.0 + v0 * v0);
            for (int iu0 = 0; iu0 < G->N_u0; iu0++)
                g_reb[(size_t(iv0) * G->N_u1 + iu1) * G->N_u0 + iu0] = row[iu0] * s;
        }
    }
}

void oracle_ramp_f64(const oracle_geom* G, double* rows, long nrows, int nthreads)
{
    // src/ramp_filter.cu:156-348: zero-pad to N_H = optimalFFTsize(2*N_u0),
    // R2C, multiply by Re(FFT(h))/N_H, C2R (unnormalized), crop.
    set_threads(nthreads);
    const int N = G->N_u0;
    const int NH = oracle_optimal_fft_size(2 * N);
    std::vector<double> h(NH);
    const float T = G->T_u0;
    for (int i = 0; i < NH; i++) {
        const float s = i < NH / 2 ? float(i) : float(i - NH);
        h[i] = double(float(1.0 / (T * kPI * (0.25 - s * s))));
    }
    std::vector<cd> Hc(NH / 2 + 1);
    r2c(h.data(), Hc.data(), NH);
    std::vector<double> Hr(NH / 2 + 1);
    for (int k = 0; k <= NH / 2; k++) Hr[k] = Hc[k].real() / double(NH);
#pragma omp parallel for schedule(static)
    for (long r = 0; r < nrows; r++) {
        std::vector<double> pad(NH, 0.0);
        std::vector<cd> spec(NH / 2 + 1);
        double* row = rows + size_t(r) * N;
        for (int i = 0; i < N; i++) pad[i] = row[i];
        r2c(pad.data(), spec.data(), NH);
        for (int k = 0; k <= NH / 2; k++) spec[k] *= Hr[k];
        c2r(spec.data(), pad.data(), NH);
        for (int i = 0; i < N; i++) row[i] = pad[i];
    }
}

void oracle_rd_gradient_f64(const double* f, double* Df, int N1, int N2, int N3, double delta, double beta,
                            int nthreads)
{
    // src/relative_differences.cu:107-173 (after clip f<1e-8 -> 0, lines 107-115)
    set_threads(nthreads);
    const size_t N = size_t(N1) * N2 * N3;
    std::vector<double> c(N);
    for (size_t i = 0; i < N; i++) c[i] = f[i] < double(0.00000001f) ? 0.0 : f[i];
    const std::vector<Nbr> nb = neighbours(false, 26);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N1; i++)
        for (int j = 0; j < N2; j++)
            for (int k = 0; k < N3; k++) {
                const double x = c[(size_t(i) * N2 + j) * N3 + k];
                double s[4] = {0, 0, 0, 0};
                for (const Nbr& n : nb) {
                    const int ii = std::min(N1 - 1, std::max(0, i + n.di));
                    const int jj = std::min(N2 - 1, std::max(0, j + n.dj));
                    const int kk = std::min(N3 - 1, std::max(0, k + n.dk));
                    s[n.cls] += drd(x, c[(size_t(ii) * N2 + jj) * N3 + kk], delta);
                }
                Df[(size_t(i) * N2 + j) * N3 + k] =
                    s[1] * dist_w(1, beta) + s[2] * dist_w(2, beta) + s[3] * dist_w(3, beta);
            }
}

double oracle_rd_cost_f64(const double* f, int N1, int N2, int N3, double delta, double beta)
{
    const size_t N = size_t(N1) * N2 * N3;
    std::vector<double> c(N);
    for (size_t i = 0; i < N; i++) c[i] = f[i] < double(0.00000001f) ? 0.0 : f[i];
    const std::vector<Nbr> nb = neighbours(false, 26);
    double total = 0.0;
    for (int i = 0; i < N1; i++)
        for (int j = 0; j < N2; j++)
            for (int k = 0; k < N3; k++) {
                const double x = c[(size_t(i) * N2 + j) * N3 + k];
                for (const Nbr& n : nb) {
                    const int ii = std::min(N1 - 1, std::max(0, i + n.di));
                    const int jj = std::min(N2 - 1, std::max(0, j + n.dj));
                    const int kk = std::min(N3 - 1, std::max(0, k + n.dk));
                    total += dist_w(n.cls, beta) * rd(x, c[(size_t(ii) * N2 + jj) * N3 + kk], delta);
                }
            }
    return total;
}

static void tv_args(double& delta, double& beta)
{
    if (beta <= 0.0) beta = 1.0;
    if (delta < 1.0e-8) delta = double(float(1.0e-8));
}

double oracle_tv_cost_f64(const double* f, int N1, int N2, int N3, double delta, double beta, double p,
                          int numNeighbors)
{
    // aTV_Huber_costTerm, src/total_variation.cu:80-201
    tv_args(delta, beta);
    const Huber hb(delta, p);
    const std::vector<Nbr> nb = neighbours(N1 == 1, numNeighbors);
    double total = 0.0;
    for (int i = 0; i < N1; i++)
        for (int j = 0; j < N2; j++)
            for (int k = 0; k < N3; k++) {
                const double x = f[(size_t(i) * N2 + j) * N3 + k];
                for (const Nbr& n : nb) {
                    const int ii = std::min(N1 - 1, std::max(0, i + n.di));
                    const int jj = std::min(N2 - 1, std::max(0, j + n.dj));
                    const int kk = std::min(N3 - 1, std::max(0, k + n.dk));
                    total += dist_w(n.cls, beta) * hb.h(x - f[(size_t(ii) * N2 + jj) * N3 + kk]);
                }
            }
    return total;
}

void oracle_tv_gradient_f64(const double* f, double* Df, int N1, int N2, int N3, double delta, double beta,
                            double p, int numNeighbors, int nthreads)
{
    // aTV_Huber_gradient, src/total_variation.cu:434-572
    set_threads(nthreads);
    tv_args(delta, beta);
    const Huber hb(delta, p);
    const std::vector<Nbr> nb = neighbours(N1 == 1, numNeighbors);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N1; i++)
        for (int j = 0; j < N2; j++)
            for (int k = 0; k < N3; k++) {
                const double x = f[(size_t(i) * N2 + j) * N3 + k];
                double s[4] = {0, 0, 0, 0};
                for (const Nbr& n : nb) {
                    const int ii = std::min(N1 - 1, std::max(0, i + n.di));
                    const int jj = std::min(N2 - 1, std::max(0, j + n.dj));
                    const int kk = std::min(N3 - 1, std::max(0, k + n.dk));
                    const double d = x - f[(size_t(ii) * N2 + jj) * N3 + kk];
                    // the reference evaluates DHuber(0) through the quadratic branch -> 0
                    s[n.cls] += hb.dh(d);
                }
                Df[(size_t(i) * N2 + j) * N3 + k] =
                    s[1] * dist_w(1, beta) + s[2] * dist_w(2, beta) + s[3] * dist_w(3, beta);
            }
}

double oracle_tv_quadform_f64(const double* f, const double* d, int N1, int N2, int N3, double delta,
                              double beta, double p, int numNeighbors)
{
    // aTV_Huber_quadFormTerm, src/total_variation.cu:218-432
    tv_args(delta, beta);
    const Huber hb(delta, p);
    const std::vector<Nbr> nb = neighbours(N1 == 1, numNeighbors);
    double total = 0.0;
    for (int i = 0; i < N1; i++)
        for (int j = 0; j < N2; j++)
            for (int k = 0; k < N3; k++) {
                const size_t o = (size_t(i) * N2 + j) * N3 + k;
                for (const Nbr& n : nb) {
                    const int ii = std::min(N1 - 1, std::max(0, i + n.di));
                    const int jj = std::min(N2 - 1, std::max(0, j + n.dj));
                    const int kk = std::min(N3 - 1, std::max(0, k + n.dk));
                    const size_t q = (size_t(ii) * N2 + jj) * N3 + kk;
                    const double dd = d[o] - d[q];
                    total += dist_w(n.cls, beta) * hb.ddh(f[o] - f[q]) * dd * dd;
                }
            }
    return total;
}

// List-mode binning, in event order: the coordinate maps of
// planogram::is_within_acceptable_angle / get_u_coords
// (src/planogram.cpp:113-141), the chest-wall shift of binning::binAcqdata
// (src/binning.cpp:630-645) and the deposit of binning::flush_queue
// (src/binning.cpp:662-790): nearest bin (linear == 0) or bilinear weights
// in (u1, u0) computed in double and added to the float bin.  The events of
// one planogram are summed in file order, as the reference's queue flushes
// do per bin.  Accumulates into g (the caller zeroes it).
void oracle_bin_events(const oracle_geom* G, const float* blue, const float* pink, long long n, float* g,
                       int linear, int chest_wall)
{
    const size_t proj = size_t(G->N_u1) * G->N_u0, obl = size_t(G->N_v0) * proj;
    const float cs = G->cos_psi, sn = G->sin_psi;
    for (long long e = 0; e < n; e++) {
        const float* b = blue + 3 * e;
        const float* q = pink + 3 * e;
        const float r0 = b[0] - q[0], r1 = b[1] - q[1], r2 = b[2] - q[2];
        const float c = -sn * r0 + cs * r1;
        if (c == 0.0f) continue;
        const float v0 = -(cs * r0 + sn * r1) / c;
        if (std::fabs(v0) > G->v_m0) continue;
        const float v1 = -r2 / c;
        if (std::fabs(v1) > G->v_m1) continue;
        const float t = b[1] * cs - b[0] * sn;
        float u1 = b[2] + v1 * t;
        const float u0 = b[0] * cs + b[1] * sn + v0 * t;
        if (chest_wall) u1 -= G->H;
        // flush_queue: slope and view by rounding in double (int(x + 0.5))
        const int iv1 = int(double((v1 - G->v1_0) / G->T_v1) + 0.5);
        if (iv1 < 0 || iv1 >= G->N_v1) continue;
        const int iv0 = int(double((v0 - G->v0_0) / G->T_v0) + 0.5);
        if (iv0 < 0 || iv0 >= G->N_v0) continue;
        float* P = g + size_t(iv1) * obl + size_t(iv0) * proj;
        const float w = 1.0f;  // the reference inserts every event with weight 1
        const float fu1 = (u1 - G->u1_0) / G->T_u1, fu0 = (u0 - G->u0_0) / G->T_u0;
        if (!linear) {
            const int a = int(double(fu1) + 0.5), bb = int(double(fu0) + 0.5);
            if (a >= 0 && a < G->N_u1 && bb >= 0 && bb < G->N_u0) P[size_t(a) * G->N_u0 + bb] += w;
            continue;
        }
        int lo1, hi1, lo0, hi0;
        float d1, d0;
        if (fu1 <= 0.0) {
            lo1 = hi1 = 0;
            d1 = 0.0f;
        } else if (fu1 >= G->N_u1 - 1) {
            lo1 = hi1 = G->N_u1 - 1;
            d1 = 0.0f;
        } else {
            lo1 = int(fu1);
            hi1 = lo1 + 1;
            d1 = fu1 - float(lo1);
        }
        if (fu0 <= 0.0) {
            lo0 = hi0 = 0;
            d0 = 0.0f;
        } else if (fu0 >= G->N_u0 - 1) {
            lo0 = hi0 = G->N_u0 - 1;
            d0 = 0.0f;
        } else {
            lo0 = int(fu0);
            hi0 = lo0 + 1;
            d0 = fu0 - float(lo0);
        }
        P[lo1 * G->N_u0 + lo0] += (1.0 - d1) * (1.0 - d0) * w;
        P[hi1 * G->N_u0 + lo0] += d1 * (1.0 - d0) * w;
        P[lo1 * G->N_u0 + hi0] += (1.0 - d1) * d0 * w;
        P[hi1 * G->N_u0 + hi0] += d1 * d0 * w;
    }
}


// ---------------------------------------------------------------------------
// Solid-angle correction (src/planogram.cpp:262-302): projection (iv1, iv0)
// is scaled by c = 2 pi (1 + v0^2 + v1^2)^1.5 / (T_v1 T_v0), the squares and
// v = i*T + start in float, the rest in double, c rounded to float; the
// inverse (the solid-angle model) uses float(1.0 / c).
// ---------------------------------------------------------------------------
float oracle_solid_angle_factor(const oracle_geom* G, int iv1, int iv0, int inverse)
{
    const float v1 = float(iv1) * G->T_v1 + G->v1_0;
    const float v0 = float(iv0) * G->T_v0 + G->v0_0;
    const double s = 1.0 + double(v0 * v0) + double(v1 * v1);
    float c = float(2.0 * 3.1415926535897932385 * std::pow(s, 1.5) / double(G->T_v1 * G->T_v0));
    if (inverse) c = float(1.0 / double(c));
    return c;
}

void oracle_solid_angle(const oracle_geom* G, float* g, int inverse)
{
    const size_t proj = size_t(G->N_u1) * G->N_u0;
    for (int iv1 = 0; iv1 < G->N_v1; iv1++)
        for (int iv0 = 0; iv0 < G->N_v0; iv0++) {
            const float c = oracle_solid_angle_factor(G, iv1, iv0, inverse);
            float* P = g + (size_t(iv1) * G->N_v0 + iv0) * proj;
            for (size_t k = 0; k < proj; k++) P[k] *= c;
        }
}

// Median of n floats (src/vector_ops.cpp:358-374): the element of rank n/2,
// and for even n the mean (in float) of the ranks n/2 and n/2 - 1.
float oracle_median(const float* x, long long n)
{
    if (n <= 0) return 0.0f;
    std::vector<float> t(x, x + n);
    std::sort(t.begin(), t.end());
    const size_t mid = size_t(n) / 2;
    if (n % 2 == 1) return t[mid];
    return (t[mid] + t[mid - 1]) / 2.0f;
}

// PETL::apply_corrections (src/petl.cpp:163-192): g = g / r (0 where r == 0,
// src/data_cube.cpp:144-149), then per projection (iv1, iv0) the bad-pixel
// in-fill of src/median_filter.cu:11-190 with threshold = rel * median(r of
// the projection):
//   outside the field of view (the projector's ray mask)  -> 0
//   r < threshold -> the median of the window's 5x5 neighbours (indices
//                    clamped at the projection's edges, so edge pixels
//                    repeat) whose divided g exceeds the threshold (the
//                    reference tests g there, not r), averaged for an even
//                    count, the mean of two for two, the one value for one,
//                    0 for none
//   otherwise      -> g / r
// Every window reads the divided values before any in-fill (the reference
// kernel rewrites g in place while other threads of the launch read it; the
// two agree whenever no window holds a pixel that the launch rewrites).
void oracle_apply_corrections(const oracle_geom* G, float* g, const float* r, float rel, int nthreads)
{
    set_threads(nthreads);
    const int N1 = G->N_u1, N0 = G->N_u0;
    const size_t proj = size_t(N1) * N0, nproj = size_t(G->N_v1) * G->N_v0;
#pragma omp parallel for schedule(dynamic)
    for (long long p = 0; p < (long long)nproj; p++) {
        const int iv1 = int(p / G->N_v0), iv0 = int(p % G->N_v0);
        float* P = g + size_t(p) * proj;
        const float* Q = r + size_t(p) * proj;
        std::vector<float> d(proj);
        for (size_t k = 0; k < proj; k++) d[k] = (Q[k] == 0.0f) ? 0.0f : P[k] / Q[k];
        const float thr = rel * oracle_median(Q, (long long)proj);
        for (int iu1 = 0; iu1 < N1; iu1++)
            for (int iu0 = 0; iu0 < N0; iu0++) {
                const size_t k = size_t(iu1) * N0 + iu0;
                if (!ray_visible(*G, iv1, iv0, iu1, iu0)) {
                    P[k] = 0.0f;
                    continue;
                }
                if (!(Q[k] < thr)) {
                    P[k] = d[k];
                    continue;
                }
                float v[25];
                int m = 0;
                for (int dj = -2; dj <= 2; dj++) {
                    const int j = tmin(tmax(iu1 + dj, 0), N1 - 1);
                    for (int dk = -2; dk <= 2; dk++) {
                        const int i = tmin(tmax(iu0 + dk, 0), N0 - 1);
                        const float x = d[size_t(j) * N0 + i];
                        if (x > thr) v[m++] = x;
                    }
                }
                if (m == 0) {
                    P[k] = 0.0f;
                } else if (m == 1) {
                    P[k] = v[0];
                } else if (m == 2) {
                    P[k] = 0.5f * (v[0] + v[1]);
                } else {
                    std::sort(v, v + m);
                    P[k] = (m % 2) ? v[m / 2] : 0.5f * (v[m / 2] + v[m / 2 - 1]);
                }
            }
    }
}


// ---------------------------------------------------------------------------
// Analytic solids, voxelization and ray tracing (src/phantom.cpp,
// src/analytic_ray_tracing_gpu.cu).
// ---------------------------------------------------------------------------

// geometricObject::init (src/phantom.cpp:535-640)
int oracle_solid_init(oracle_solid* s, int type, const float* c, const float* r, float val, const float* A,
                      const float* clip)
{
    std::memset(s, 0, sizeof(*s));
    s->type = -1;
    if (!c || !r || type < 0 || type > 7) return 0;
    s->type = type;
    for (int i = 0; i < 3; i++) {
        s->centers[i] = s->given_c[i] = c[i];
        s->radii[i] = s->given_r[i] = r[i];
    }
    if (clip) {
        for (int i = 0; i < 3; i++)
            if (clip[i] != 0.0) {
                s->clip[s->num_clip][i] = -1.0f;
                s->clip[s->num_clip][3] = -clip[i];
                s->num_clip += 1;
            }
    }
    s->val = val;
    if (A) {
        for (int i = 0; i < 9; i++) {
            s->A[i] = A[i];
            if (i == 0 || i == 4 || i == 8) {
                if (std::fabs(A[i] - 1.0) > 1.0e-8) s->rotated = 1;
            } else if (std::fabs(A[i]) > 1.0e-8) {
                s->rotated = 1;
            }
        }
    }
    auto cone = [&](int axis, int a, int b, float* cc, float* rr, float* clip_cone) {
        // axis length l and end radii r_1 (index a), r_2 (index b)
        const double l = rr[axis], r_1 = rr[a], r_2 = rr[b];
        rr[a] = float(std::fabs(r_2 - r_1) / (2.0 * l));
        rr[b] = rr[a];
        rr[axis] = 1.0f;
        cc[axis] = float(cc[axis] - l * (r_2 + r_1) / (r_2 - r_1));
        clip_cone[0] = float(-l + l * (r_2 + r_1) / (r_2 - r_1));
        clip_cone[1] = float(l + l * (r_2 + r_1) / (r_2 - r_1));
    };
    if (type == 5) cone(0, 1, 2, s->centers, s->radii, s->clip_cone);
    if (type == 6) cone(1, 0, 2, s->centers, s->radii, s->clip_cone);
    if (type == 7) cone(2, 0, 1, s->centers, s->radii, s->clip_cone);
    return 1;
}

namespace {

// phantom::isInside (src/phantom.cpp:337-387)
bool vox_is_inside(float x, float y, float z, int type, const float* clip, const float* cone)
{
    bool in = false;
    switch (type) {
    case 0: in = x * x + y * y + z * z <= 1.0; break;
    case 1: in = std::fabs(x) <= 1.0 && std::fabs(y) <= 1.0 && std::fabs(z) <= 1.0; break;
    case 2: in = std::fabs(x) <= 1.0 && y * y + z * z <= 1.0; break;
    case 3: in = std::fabs(y) <= 1.0 && x * x + z * z <= 1.0; break;
    case 4: in = std::fabs(z) <= 1.0 && x * x + y * y <= 1.0; break;
    case 5: in = y * y + z * z <= x * x && cone[0] <= x && x <= cone[1]; break;
    case 6: in = x * x + z * z <= y * y && cone[0] <= y && y <= cone[1]; break;
    case 7: in = x * x + y * y <= z * z && cone[0] <= z && z <= cone[1]; break;
    default: break;
    }
    if (clip) {
        if (clip[0] * x > 0.0) in = false;
        if (clip[1] * y > 0.0) in = false;
        if (clip[2] * z > 0.0) in = false;
    }
    return in;
}

// phantom::addObject(f, ...) for one solid (src/phantom.cpp:141-335),
// with c and r as the voxelizer passes them
void vox_add(float* f, int numX, int numY, int numZ, float T_x, float T_z, float x_0, float y_0, float z_0, int type,
             float* c, float* r, float val, const float* A, const float* clip, int os)
{
    const float T_y = T_x;
    auto xi = [&](float v) { return (v - x_0) / T_x; };
    auto yi = [&](float v) { return (v - y_0) / T_y; };
    auto zi = [&](float v) { return (v - z_0) / T_z; };
    int minX = int(std::floor(xi(c[0] - r[0] - T_x))), maxX = int(std::ceil(xi(c[0] + r[0] + T_x)));
    int minY = int(std::floor(yi(c[1] - r[1] - T_y))), maxY = int(std::ceil(yi(c[1] + r[1] + T_y)));
    int minZ = int(std::floor(zi(c[2] - r[2] - T_z))), maxZ = int(std::ceil(zi(c[2] + r[2] + T_z)));
    const bool rotated = A && (A[0] != 1.0 || A[4] != 1.0 || A[8] != 1.0);
    if (rotated || (type >= 5 && type <= 7)) {
        const float r_max = std::sqrt(3.0) * std::max(r[0], std::max(r[1], r[2]));
        minX = int(std::floor(xi(c[0] - r_max - T_x)));
        maxX = int(std::ceil(xi(c[0] + r_max + T_x)));
        minY = int(std::floor(yi(c[1] - r_max - T_y)));
        maxY = int(std::ceil(yi(c[1] + r_max + T_y)));
        minZ = int(std::floor(zi(c[2] - r_max - T_z)));
        maxZ = int(std::ceil(zi(c[2] + r_max + T_z)));
    }
    float cone[2] = {0.0f, 0.0f};
    auto conify = [&](int axis, int a, int b) {
        const double l = r[axis], r_1 = r[a], r_2 = r[b];
        r[a] = std::fabs(r_2 - r_1) / (2.0 * l);
        r[b] = r[a];
        r[axis] = 1.0;
        c[axis] = c[axis] - l * (r_2 + r_1) / (r_2 - r_1);
        cone[0] = -l + l * (r_2 + r_1) / (r_2 - r_1);
        cone[1] = l + l * (r_2 + r_1) / (r_2 - r_1);
    };
    if (type == 5) conify(0, 1, 2);
    if (type == 6) conify(1, 0, 2);
    if (type == 7) conify(2, 0, 1);
    auto clampi = [](int v, int n) { return std::max(0, std::min(n - 1, v)); };
    minX = clampi(minX, numX), maxX = clampi(maxX, numX);
    minY = clampi(minY, numY), maxY = clampi(maxY, numY);
    minZ = clampi(minZ, numZ), maxZ = clampi(maxZ, numZ);
    os = std::max(1, std::min(os, 5));
    auto inside = [&](float x, float y, float z) {
        if (rotated) {
            const float xr = (A[0] * (x - c[0]) + A[1] * (y - c[1]) + A[2] * (z - c[2])) / r[0];
            const float yr = (A[3] * (x - c[0]) + A[4] * (y - c[1]) + A[5] * (z - c[2])) / r[1];
            const float zr = (A[6] * (x - c[0]) + A[7] * (y - c[1]) + A[8] * (z - c[2])) / r[2];
            return vox_is_inside(xr, yr, zr, type, clip, cone);
        }
        return vox_is_inside((x - c[0]) / r[0], (y - c[1]) / r[1], (z - c[2]) / r[2], type, clip, cone);
    };
#pragma omp parallel for
    for (int iz = minZ; iz <= maxZ; iz++) {
        const float z = iz * T_z + z_0;
        for (int iy = minY; iy <= maxY; iy++) {
            const float y = iy * T_y + y_0;
            float* line = f + (size_t(iz) * numY + iy) * numX;
            for (int ix = minX; ix <= maxX; ix++) {
                const float x = ix * T_x + x_0;
                if (os == 1) {
                    if (inside(x, y, z)) line[ix] = val;
                    continue;
                }
                const double frac = 1.0 / float(os * os * os);
                const float cur = line[ix];
                float acc = 0.0;
                for (int kz = 0; kz < os; kz++) {
                    const float zs = z + T_z / float(os + 1) * (float(kz) - 0.5 * float(os - 1));
                    for (int ky = 0; ky < os; ky++) {
                        const float ys = y + T_y / float(os + 1) * (float(ky) - 0.5 * float(os - 1));
                        for (int kx = 0; kx < os; kx++) {
                            const float xs = x + T_x / float(os + 1) * (float(kx) - 0.5 * float(os - 1));
                            if (inside(xs, ys, zs)) acc += (val - cur) * frac;
                        }
                    }
                }
                line[ix] = acc + cur;
            }
        }
    }
}

const float kOOB = 1.0e12f;  // src/analytic_ray_tracing_gpu.cu:21

// src/analytic_ray_tracing_gpu.cu:84-114
bool rt_slab(float* ts, float p, float r)
{
    if (std::fabs(r) < 1e-12f) {
        if (std::fabs(p) < 1.0f) {
            ts[0] = -kOOB;
            ts[1] = kOOB;
            return true;
        }
        return false;
    }
    if (r > 0.0f) {
        ts[0] = (-1.0f - p) / r;
        ts[1] = (1.0f - p) / r;
    } else {
        ts[1] = (-1.0f - p) / r;
        ts[0] = (1.0f - p) / r;
    }
    return true;
}

// src/analytic_ray_tracing_gpu.cu:150-463
bool rt_normalized(const double* p, const double* r, float* ts, const oracle_solid& sd)
{
    ts[0] = ts[1] = -kOOB;
    const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double pr = r[0] * p[0] + r[1] * p[1] + r[2] * p[2];
    auto quad2 = [&](double b, double a, double c, float* t) {  // b^2 - a c > 0 -> roots
        double disc = b * b - a * c;
        if (!(disc > 0.0)) return false;
        disc = std::sqrt(disc);
        t[0] = float((-b - disc) / a);
        t[1] = float((-b + disc) / a);
        return true;
    };
    float tz[2], t[2];
    switch (sd.type) {
    case 0: {
        double disc = pr * pr + rr * (1.0 - (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
        if (!(disc > 0.0)) return false;
        disc = std::sqrt(disc);
        ts[0] = float((-pr - disc) / rr);
        ts[1] = float((-pr + disc) / rr);
        break;
    }
    case 1: {
        float tx[2], ty[2];
        if (!rt_slab(tx, float(p[0]), float(r[0])) || !rt_slab(ty, float(p[1]), float(r[1])) ||
            !rt_slab(tz, float(p[2]), float(r[2])))
            return false;
        ts[0] = std::max(std::max(tx[0], ty[0]), tz[0]);
        ts[1] = std::min(std::min(tx[1], ty[1]), tz[1]);
        break;
    }
    case 4: case 2: case 3: {
        int k, i, j;
        double b, c;
        const double a = sd.type == 4 ? rr - r[2] * r[2] : sd.type == 2 ? rr - r[0] * r[0] : rr - r[1] * r[1];
        if (sd.type == 4) {
            k = 2, i = 0, j = 1;
            b = pr - p[2] * r[2];
            c = p[0] * p[0] + p[1] * p[1] - 1.0;
        } else if (sd.type == 2) {
            k = 0, i = 1, j = 2;
            b = p[2] * r[2] + p[1] * r[1];
            c = p[2] * p[2] + p[1] * p[1] - 1.0;
        } else {
            k = 1, i = 0, j = 2;
            b = p[0] * r[0] + p[2] * r[2];
            c = p[0] * p[0] + p[2] * p[2] - 1.0;
        }
        if (quad2(b, a, c, t)) {
            if (!rt_slab(tz, float(p[k]), float(r[k]))) return false;
            ts[0] = std::max(t[0], tz[0]);
            ts[1] = std::min(t[1], tz[1]);
        } else if (r[i] == 0.0 && r[j] == 0.0 && p[i] * p[i] + p[j] * p[j] <= 1.0) {
            if (!rt_slab(ts, float(p[k]), float(r[k]))) return false;
        } else {
            return false;
        }
        break;
    }
    case 7: case 5: {
        const int k = sd.type == 7 ? 2 : 0, i = sd.type == 7 ? 0 : 2, j = 1;
        const double a = r[i] * r[i] + r[j] * r[j] - r[k] * r[k];
        const double b = p[i] * r[i] + p[j] * r[j] - p[k] * r[k];
        const double c = p[i] * p[i] + p[j] * p[j] - p[k] * p[k];
        if (!quad2(b, a, c, t)) return false;
        if (t[0] > t[1]) std::swap(t[0], t[1]);
        const double shift = 0.5 * (sd.clip_cone[1] + sd.clip_cone[0]);
        const double scale = 0.5 * (sd.clip_cone[1] - sd.clip_cone[0]);
        if (!rt_slab(tz, float((p[k] - shift) / scale), float(r[k] / scale))) return false;
        ts[0] = std::max(t[0], tz[0]);
        ts[1] = std::min(t[1], tz[1]);
        break;
    }
    case 6: {
        const double a = r[0] * r[0] + r[2] * r[2] - r[1] * r[1];
        const double b = p[0] * r[0] + p[2] * r[2] - p[1] * r[1];
        const double c = p[0] * p[0] + p[2] * p[2] - p[1] * p[1];
        double disc = b * b - a * c;
        if (!(disc > 0.0)) break;
        disc = std::sqrt(disc);
        double tmin = (-b - disc) / a, tmax = (-b + disc) / a;
        if (tmin > tmax) std::swap(tmin, tmax);
        const double shift = 0.5 * (sd.clip_cone[1] + sd.clip_cone[0]);
        const double scale = 0.5 * (sd.clip_cone[1] - sd.clip_cone[0]);
        if (!rt_slab(tz, float((p[1] - shift) / scale), float(r[1] / scale))) break;
        if (!(std::fabs(r[1]) > 1.0e-12f)) {
            ts[0] = float(tmin);
            ts[1] = float(tmax);
            break;
        }
        auto in_at = [&](float tt) {
            double x = p[0] + tt * r[0], y = p[1] + tt * r[1], z = p[2] + tt * r[2];
            return x * x + z * z <= y * y;
        };
        const bool in0 = in_at(tz[0]), in1 = in_at(tz[1]);
        if (in0 && in1) {
            ts[0] = tz[0];
            ts[1] = tz[1];
        } else if (in0) {
            ts[0] = tz[0];
            ts[1] = float((tz[0] <= tmin && tmin <= tz[1]) ? tmin : tmax);
        } else if (in1) {
            ts[0] = float((tz[0] <= tmin && tmin <= tz[1]) ? tmin : tmax);
            ts[1] = tz[1];
        } else if (tz[0] <= tmin && tmax <= tz[1]) {
            ts[0] = float(tmin);
            ts[1] = float(tmax);
        } else {
            ts[0] = ts[1] = -kOOB;
            return false;
        }
        break;
    }
    default:
        return false;
    }
    if (ts[0] >= ts[1]) {
        ts[0] = ts[1] = -kOOB;
        return false;
    }
    return true;
}

// src/analytic_ray_tracing_gpu.cu:465-518 (with the clipping planes,
// 116-148)
bool rt_hit(const float* p, const float* r, float* ts, const oracle_solid& sd)
{
    double q[3], m[3];
    if (!sd.rotated) {
        for (int k = 0; k < 3; k++) {
            q[k] = (p[k] - sd.centers[k]) / sd.radii[k];
            m[k] = r[k] / sd.radii[k];
        }
    } else {
        const double d[3] = {p[0] - sd.centers[0], p[1] - sd.centers[1], p[2] - sd.centers[2]};
        for (int k = 0; k < 3; k++) {
            q[k] = (d[0] * sd.A[3 * k] + d[1] * sd.A[3 * k + 1] + d[2] * sd.A[3 * k + 2]) / sd.radii[k];
            m[k] = (r[0] * sd.A[3 * k] + r[1] * sd.A[3 * k + 1] + r[2] * sd.A[3 * k + 2]) / sd.radii[k];
        }
    }
    if (!rt_normalized(q, m, ts, sd)) return false;
    for (int i = 0; i < sd.num_clip; i++) {
        const float* n = sd.clip[i];
        const float pn = n[0] * p[0] + n[1] * p[1] + n[2] * p[2];
        const float rn = n[0] * r[0] + n[1] * r[1] + n[2] * r[2];
        if (std::fabs(rn) < 1.0e-12f) {
            if (pn < n[3]) return false;
        } else if (rn > 0.0f) {
            const float t = (n[3] - pn) / rn;
            if (ts[1] < t) return false;
            if (t > ts[0]) ts[0] = t;
        } else {
            const float t = (n[3] - pn) / rn;
            if (ts[0] > t) return false;
            if (ts[1] > t) ts[1] = t;
        }
    }
    return ts[1] > ts[0];
}

// src/analytic_ray_tracing_gpu.cu:536-691: line integral (split == 0) or
// the two half-lines (*fwd, *bwd)
void rt_line(const oracle_solid* sd, int n, const float* p, const float* r, int split, float* fwd, float* bwd)
{
    std::vector<float> ends, t0(n), t1(n);
    std::vector<int> idx;
    for (int i = 0; i < n; i++) {
        float ts[2];
        if (rt_hit(p, r, ts, sd[i])) {
            ends.push_back(ts[0]);
            ends.push_back(ts[1]);
            t0[i] = ts[0];
            t1[i] = ts[1];
            idx.push_back(i);
        }
    }
    *fwd = *bwd = 0.0f;
    std::sort(ends.begin(), ends.end());
    for (int i = 0; i + 1 < int(ends.size()); i++) {
        const float mid = (ends[i + 1] + ends[i]) * 0.5f;
        for (int h = int(idx.size()) - 1; h >= 0; h--) {
            const int j = idx[h];
            if (t0[j] <= mid && mid <= t1[j]) {
                const float v = sd[j].val * (ends[i + 1] - ends[i]);
                if (!split || mid >= 0.0f)
                    *fwd += v;
                else
                    *bwd += v;
                break;
            }
        }
    }
}

}  // namespace

// phantom::voxelize (src/phantom.cpp:105-139): every solid in order
void oracle_voxelize(const oracle_solid* sd, int n, float* f, int numX, int numY, int numZ, float T_x, float T_z,
                     float x_0, float y_0, float z_0, int os)
{
    for (int k = 0; k < n; k++) {
        float c[3], r[3], clip[4];
        const bool cone = sd[k].type >= 5 && sd[k].type <= 7;
        for (int i = 0; i < 3; i++) {
            c[i] = cone ? sd[k].given_c[i] : sd[k].centers[i];
            r[i] = cone ? sd[k].given_r[i] : sd[k].radii[i];
        }
        for (int i = 0; i < 4; i++) clip[i] = -sd[k].clip[0][i];
        const float* cp = (!cone && sd[k].num_clip > 0) ? clip : nullptr;
        vox_add(f, numX, numY, numZ, T_x, T_z, x_0, y_0, z_0, sd[k].type, c, r, sd[k].val, sd[k].A, cp, os);
    }
}

// rayTracingKernel / stoppingPowerKernel (src/analytic_ray_tracing_gpu.cu:
// 693-846) for one planogram, with the direction and field-of-view rules of
// the kernels (cos/sin of the float psi in float)
void oracle_ray_trace(const oracle_geom* G, const oracle_solid* sd, int n, float* g, int oversampling, int stopping,
                      int nthreads)
{
    set_threads(nthreads);
    int os = std::max(1, std::min(oversampling, 11));
    if (os % 2 == 0) os += 1;
    os = std::max(1, std::min(os, 11));
    const float cs = std::cos(G->psi), sn = std::sin(G->psi);
    const long long total = (long long)G->N_v1 * G->N_v0 * G->N_u1 * G->N_u0;
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long id = 0; id < total; id++) {
        long long t = id;
        const int iu0 = int(t % G->N_u0);
        t /= G->N_u0;
        const int iu1 = int(t % G->N_u1);
        t /= G->N_u1;
        const int iv0 = int(t % G->N_v0), iv1 = int(t / G->N_v0);
        const float v1 = std::fma(float(iv1), G->T_v1, G->v1_0);
        const float v0 = std::fma(float(iv0), G->T_v0, G->v0_0);
        const float u1 = std::fma(float(iu1), G->T_u1, G->u1_0);
        const float u0 = std::fma(float(iu0), G->T_u0, G->u0_0);
        if (std::fabs(u1) - 0.5f * G->T_u1 > std::fma(-G->R, std::fabs(v1), G->H) ||
            std::fabs(u0) - 0.5f * G->T_v0 > std::fma(G->R, std::fabs(v0), G->L)) {
            g[id] = 0.0f;
            continue;
        }
        float r[3] = {-(v0 * cs + sn), -(v0 * sn - cs), -v1};
        const float mag = 1.0f / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        for (int k = 0; k < 3; k++) r[k] = r[k] / mag;
        auto value = [&](float du1, float du0) {
            const float w = u0 + du0;
            const float p[3] = {w * cs, w * sn, u1 + du1};
            float fwd, bwd;
            rt_line(sd, n, p, r, stopping, &fwd, &bwd);
            return stopping ? (1.0f - std::exp(-fwd)) * (1.0f - std::exp(-bwd)) : fwd;
        };
        if (os <= 1) {
            g[id] = value(0.0f, 0.0f);
        } else {
            const float d1 = G->T_u1 / float(os + 1), d0 = G->T_u0 / float(os + 1);
            const int rad = (os - 1) / 2;
            float acc = 0.0f;
            for (int j = -rad; j <= rad; j++)
                for (int k = -rad; k <= rad; k++) acc += value(j * d1, k * d0);
            g[id] = acc / float(os * os);
        }
    }
}

}  // extern "C"
