// Analytic phantoms: the solids of a phantom or of a detector-module model,
// their voxelization, and analytic ray tracing of planograms through them
// (line integrals, or the detector stopping power of each coincidence line).
//
// Solids (src/phantom.cpp:487-640): ellipsoids, parallelepipeds, cylinders
// and cones along x, y or z, each with a centre, radii, a value, an optional
// rotation and optional clipping planes.
//
// voxelize (src/phantom.cpp:105-335, host code in the reference): one thread
// per voxel applies the solids in order (later solids replace earlier
// values); the float and double operations are rounding-pinned to the
// reference's host arithmetic, so the volume is bit-exact.
//
// ray tracing (src/analytic_ray_tracing_gpu.cu:48-846): one thread per
// planogram bin.  Each solid's entry and exit parameters along the bin's line
// are found in the solid's normalised frame; the end points are sorted and
// each interval between consecutive end points is credited to the last solid
// (in insertion order) that covers its midpoint.  The solids are staged in
// shared memory with a padded axis-aligned box each, grouped into clusters of
// up to 8 nearby solids with a box around each cluster; a line tests a
// cluster's box, then the boxes of its members, and runs the exact
// intersection only for the solids whose box it meets (conservative tests:
// the result is unchanged).  The hits of a line are kept per thread
// (up to kMaxHits; a line with more is resolved by rescanning the solids per
// interval, which gives the same sum).  The reference's line parameterisation is kept: its
// direction is the unnormalised direction times its own length (the
// reference divides by rsqrt of the squared length), so lengths come out
// divided by 1 + v0^2 + v1^2; and its field-of-view test for u0 uses half
// of T_v0 (src/analytic_ray_tracing_gpu.cu:721).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"

namespace petl {
namespace {

enum SolidType { kEllipsoid = 0, kBox = 1, kCylX = 2, kCylY = 3, kCylZ = 4, kConeX = 5, kConeY = 6, kConeZ = 7 };

constexpr float kFar = 1.0e12f;  // parameter of an unbounded side
constexpr int kMaxHits = 32;     // hits of one line kept per thread
constexpr int kRayThreads = 128;
constexpr int kSmemSolids = 176;  // solids, boxes, clusters staged in shared memory (<= 45 KB)

// ---------------------------------------------------------------------------
// intersections (device)
// ---------------------------------------------------------------------------

// Parameters where p + t r crosses -1 and +1 (float arithmetic); a line
// parallel to the slab is unbounded inside it and misses outside.
__device__ __forceinline__ bool slab(float p, float r, float& t0, float& t1)
{
    if (fabsf(r) < 1e-12f) {
        if (fabsf(p) < 1.0f) {
            t0 = -kFar;
            t1 = kFar;
            return true;
        }
        return false;
    }
    const float a = (-1.0f - p) / r, b = (1.0f - p) / r;
    t0 = r > 0.0f ? a : b;
    t1 = r > 0.0f ? b : a;
    return true;
}

// Quadric roots of a t^2 + 2 b t + c = 0 as floats, if the discriminant is
// positive.
__device__ __forceinline__ bool roots(double a, double b_half, double c, float& t0, float& t1)
{
    double disc = b_half * b_half - a * c;
    if (!(disc > 0.0)) return false;
    disc = sqrt(disc);
    t0 = float((-b_half - disc) / a);
    t1 = float((-b_half + disc) / a);
    return true;
}

// Entry/exit parameters of the line q + t m with the solid in its normalised
// frame (src/analytic_ray_tracing_gpu.cu:150-463).  Axis k is the solid's
// axis for cylinders and cones; i, j the other two.
__device__ bool normalized_hit(const petl_solid& s, const double q[3], const double m[3], float& t0, float& t1)
{
    t0 = -kFar;
    t1 = -kFar;
    const double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    const double qm = m[0] * q[0] + m[1] * q[1] + m[2] * q[2];
    switch (s.type) {
    case kEllipsoid: {
        double disc = qm * qm + mm * (1.0 - (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
        if (!(disc > 0.0)) return false;
        disc = sqrt(disc);
        t0 = float((-qm - disc) / mm);
        t1 = float((-qm + disc) / mm);
        break;
    }
    case kBox: {
        float a0, a1, b0, b1, c0, c1;
        if (!slab(float(q[0]), float(m[0]), a0, a1) || !slab(float(q[1]), float(m[1]), b0, b1) ||
            !slab(float(q[2]), float(m[2]), c0, c1))
            return false;
        t0 = fmaxf(fmaxf(a0, b0), c0);
        t1 = fminf(fminf(a1, b1), c1);
        break;
    }
    case kCylX:
    case kCylY:
    case kCylZ: {
        // the reference's term order per axis (src/analytic_ray_tracing_gpu.cu:205-281)
        const int k = s.type - kCylX, i = k == 0 ? 1 : 0, j = k == 2 ? 1 : 2;
        const double mm2 = mm - m[k] * m[k];
        double qm2, cc;
        if (k == 2) {
            qm2 = qm - q[2] * m[2];
            cc = q[0] * q[0] + q[1] * q[1] - 1.0;
        } else if (k == 0) {
            qm2 = q[2] * m[2] + q[1] * m[1];
            cc = q[2] * q[2] + q[1] * q[1] - 1.0;
        } else {
            qm2 = q[0] * m[0] + q[2] * m[2];
            cc = q[0] * q[0] + q[2] * q[2] - 1.0;
        }
        float a0, a1, z0, z1;
        if (roots(mm2, qm2, cc, a0, a1)) {
            if (!slab(float(q[k]), float(m[k]), z0, z1)) return false;
            t0 = fmaxf(a0, z0);
            t1 = fminf(a1, z1);
        } else if (m[i] == 0.0 && m[j] == 0.0 && q[i] * q[i] + q[j] * q[j] <= 1.0) {
            if (!slab(float(q[k]), float(m[k]), t0, t1)) return false;
        } else {
            return false;
        }
        break;
    }
    case kConeX:
    case kConeZ: {
        const int k = s.type == kConeX ? 0 : 2, i = k == 0 ? 2 : 0, j = 1;
        const double a = m[i] * m[i] + m[j] * m[j] - m[k] * m[k];
        const double b = q[i] * m[i] + q[j] * m[j] - q[k] * m[k];
        const double c = q[i] * q[i] + q[j] * q[j] - q[k] * q[k];
        float a0, a1, z0, z1;
        if (!roots(a, b, c, a0, a1)) return false;
        if (a0 > a1) {
            const float t = a0;
            a0 = a1;
            a1 = t;
        }
        const double shift = 0.5 * double(s.clip_cone[1] + s.clip_cone[0]);
        const double scale = 0.5 * double(s.clip_cone[1] - s.clip_cone[0]);
        if (!slab(float((q[k] - shift) / scale), float(m[k] / scale), z0, z1)) return false;
        t0 = fmaxf(a0, z0);
        t1 = fminf(a1, z1);
        break;
    }
    case kConeY: {
        // the y cone also tells the nappe it is clipped to from the end
        // points of its axial slab (src/analytic_ray_tracing_gpu.cu:352-455)
        const double a = m[0] * m[0] + m[2] * m[2] - m[1] * m[1];
        const double b = q[0] * m[0] + q[2] * m[2] - q[1] * m[1];
        const double c = q[0] * q[0] + q[2] * q[2] - q[1] * q[1];
        double disc = b * b - a * c;
        if (!(disc > 0.0)) break;
        disc = sqrt(disc);
        double lo = (-b - disc) / a, hi = (-b + disc) / a;
        if (lo > hi) {
            const double t = lo;
            lo = hi;
            hi = t;
        }
        const double shift = 0.5 * double(s.clip_cone[1] + s.clip_cone[0]);
        const double scale = 0.5 * double(s.clip_cone[1] - s.clip_cone[0]);
        float z0, z1;
        if (!slab(float((q[1] - shift) / scale), float(m[1] / scale), z0, z1)) break;
        if (!(fabs(m[1]) > double(1.0e-12f))) {
            t0 = float(lo);
            t1 = float(hi);
            break;
        }
        auto inside = [&](float t) {
            const double x = q[0] + double(t) * m[0], y = q[1] + double(t) * m[1], z = q[2] + double(t) * m[2];
            return x * x + z * z <= y * y;
        };
        const bool in0 = inside(z0), in1 = inside(z1);
        const bool lo_in = double(z0) <= lo && lo <= double(z1);
        if (in0 && in1) {
            t0 = z0;
            t1 = z1;
        } else if (in0) {
            t0 = z0;
            t1 = float(lo_in ? lo : hi);
        } else if (in1) {
            t0 = float(lo_in ? lo : hi);
            t1 = z1;
        } else if (double(z0) <= lo && hi <= double(z1)) {
            t0 = float(lo);
            t1 = float(hi);
        } else {
            t0 = t1 = -kFar;
            return false;
        }
        break;
    }
    default:
        return false;
    }
    if (t0 >= t1) {
        t0 = t1 = -kFar;
        return false;
    }
    return true;
}

// Entry/exit parameters of the line p + t r with a solid
// (src/analytic_ray_tracing_gpu.cu:465-518): move to the solid's frame
// (shift, rotate, scale by the radii), intersect, then apply the clipping
// planes in world coordinates.
__device__ bool solid_hit(const petl_solid& s, float3 p, float3 r, float& t0, float& t1)
{
    double q[3], m[3];
    if (!s.rotated) {
        q[0] = (p.x - s.centers[0]) / s.radii[0];
        q[1] = (p.y - s.centers[1]) / s.radii[1];
        q[2] = (p.z - s.centers[2]) / s.radii[2];
        m[0] = r.x / s.radii[0];
        m[1] = r.y / s.radii[1];
        m[2] = r.z / s.radii[2];
    } else {
        const double d[3] = {p.x - s.centers[0], p.y - s.centers[1], p.z - s.centers[2]};
        for (int k = 0; k < 3; k++) {
            q[k] = (d[0] * s.A[3 * k] + d[1] * s.A[3 * k + 1] + d[2] * s.A[3 * k + 2]) / s.radii[k];
            m[k] = (r.x * s.A[3 * k] + r.y * s.A[3 * k + 1] + r.z * s.A[3 * k + 2]) / s.radii[k];
        }
    }
    if (!normalized_hit(s, q, m, t0, t1)) return false;
    for (int i = 0; i < s.num_clip; i++) {
        const float* c = s.clip[i];
        const float pn = c[0] * p.x + c[1] * p.y + c[2] * p.z;
        const float rn = c[0] * r.x + c[1] * r.y + c[2] * r.z;
        if (fabsf(rn) < 1.0e-12f) {
            if (pn < c[3]) {
                t0 = t1 = -kFar;
                return false;
            }
            continue;
        }
        const float t = (c[3] - pn) / rn;
        if (rn > 0.0f) {
            if (t1 < t) {
                t0 = t1 = -kFar;
                return false;
            }
            t0 = fmaxf(t0, t);
        } else {
            if (t0 > t) {
                t0 = t1 = -kFar;
                return false;
            }
            t1 = fminf(t1, t);
        }
    }
    return t1 > t0;
}

// Axis-aligned box around a solid for culling, padded (always != 0: the
// solid is always tested).
struct Bound {
    float lo[3], hi[3];
    int always, pad;
};

// Whether the line p + t r may meet the solid: the line against the padded
// box by slabs (inv = 1 / r per axis, infinite for a zero component).  The
// padding (1e-4 of the extent plus 1e-3) exceeds the float error of the
// slab parameters, so every line the exact test accepts passes.
__device__ __forceinline__ bool may_hit(const Bound& b, float3 p, float3 inv)
{
    if (b.always) return true;
    const float ax = (b.lo[0] - p.x) * inv.x, bx = (b.hi[0] - p.x) * inv.x;
    const float ay = (b.lo[1] - p.y) * inv.y, by = (b.hi[1] - p.y) * inv.y;
    const float az = (b.lo[2] - p.z) * inv.z, bz = (b.hi[2] - p.z) * inv.z;
    const float tmin = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    const float tmax = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
    return tmin <= tmax;
}

// A group of up to kClusterSize solids that lie close together: the padded
// box around all of them, and their indices order[first .. first + count).
struct Cluster {
    Bound box;
    int first, count, pad0, pad1;
};

constexpr int kClusterSize = 8;

struct LineSums {
    float fwd, bwd;  // value x length with the interval midpoint at t >= 0 / t < 0
};

// Sum of value x length along p + t r: end points sorted, each interval
// credited to the last solid covering its midpoint
// (src/analytic_ray_tracing_gpu.cu:536-691).  SPLIT: the two half-lines
// apart (stopping power); otherwise every interval into fwd, in order.
template <bool SPLIT>
__device__ LineSums line_sums(const petl_solid* solids, const Bound* bounds, const Cluster* clusters, int ncl,
                              const int* order, int n, float3 p, float3 r)
{
    float h0[kMaxHits], h1[kMaxHits], e[2 * kMaxHits];
    int hid[kMaxHits];
    int count = 0;
    bool overflow = false;
    const float3 inv = make_float3(1.0f / r.x, 1.0f / r.y, 1.0f / r.z);
    // clusters, then their members; the hits are kept in solid order
    for (int c = 0; c < ncl && !overflow; c++) {
        const Cluster& cl = clusters[c];
        if (!may_hit(cl.box, p, inv)) continue;
        for (int k = cl.first; k < cl.first + cl.count; k++) {
            const int j = order[k];
            float t0, t1;
            if (!may_hit(bounds[j], p, inv) || !solid_hit(solids[j], p, r, t0, t1)) continue;
            if (count == kMaxHits) {
                overflow = true;
                break;
            }
            int pos = count;
            while (pos > 0 && hid[pos - 1] > j) {
                h0[pos] = h0[pos - 1];
                h1[pos] = h1[pos - 1];
                hid[pos] = hid[pos - 1];
                pos--;
            }
            h0[pos] = t0;
            h1[pos] = t1;
            hid[pos] = j;
            e[2 * count] = t0;
            e[2 * count + 1] = t1;
            count++;
        }
    }
    LineSums acc{0.0f, 0.0f};
    if (!overflow) {
        const int ne = 2 * count;
        for (int a = 1; a < ne; a++) {
            const float x = e[a];
            int b = a - 1;
            while (b >= 0 && e[b] > x) {
                e[b + 1] = e[b];
                b--;
            }
            e[b + 1] = x;
        }
        for (int i = 0; i + 1 < ne; i++) {
            const float mid = (e[i + 1] + e[i]) * 0.5f;
            for (int h = count - 1; h >= 0; h--)
                if (h0[h] <= mid && mid <= h1[h]) {
                    const float v = solids[hid[h]].val * (e[i + 1] - e[i]);
                    if (!SPLIT || mid >= 0.0f)
                        acc.fwd += v;
                    else
                        acc.bwd += v;
                    break;
                }
        }
        return acc;
    }
    // more hits than kept: walk the distinct end points in order, rescanning
    // the solids (zero-length intervals add nothing, so the sum is the same)
    float cur = kFar * 4.0f;
    for (int j = 0; j < n; j++) {
        float t0, t1;
        if (solid_hit(solids[j], p, r, t0, t1)) cur = fminf(cur, t0);
    }
    for (;;) {
        float next = kFar * 4.0f;
        for (int j = 0; j < n; j++) {
            float t0, t1;
            if (!solid_hit(solids[j], p, r, t0, t1)) continue;
            if (t0 > cur) next = fminf(next, t0);
            if (t1 > cur) next = fminf(next, t1);
        }
        if (next == kFar * 4.0f) break;
        const float mid = (next + cur) * 0.5f;
        for (int j = n - 1; j >= 0; j--) {
            float t0, t1;
            if (solid_hit(solids[j], p, r, t0, t1) && t0 <= mid && mid <= t1) {
                const float v = solids[j].val * (next - cur);
                if (!SPLIT || mid >= 0.0f)
                    acc.fwd += v;
                else
                    acc.bwd += v;
                break;
            }
        }
        cur = next;
    }
    return acc;
}

struct RayArgs {
    petl_geom G;
    const petl_solid* solids;
    const Bound* bounds;
    const Cluster* clusters;
    const int* order;
    int ncl;
    int n;
    float* g;
    int os;
    float cos_psi, sin_psi;
    long long total;
};

template <bool STOP>
__global__ void __launch_bounds__(kRayThreads) k_ray_trace(const RayArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const bool staged = a.n <= kSmemSolids;
    Cluster* sc = reinterpret_cast<Cluster*>(smem_raw);
    Bound* sb = reinterpret_cast<Bound*>(sc + (staged ? a.ncl : 0));
    petl_solid* ss = reinterpret_cast<petl_solid*>(sb + (staged ? a.n : 0));
    int* so = reinterpret_cast<int*>(ss + (staged ? a.n : 0));
    if (staged) {
        auto copy = [&](void* dst, const void* src, int words) {
            for (int i = threadIdx.x; i < words; i += blockDim.x)
                static_cast<int*>(dst)[i] = static_cast<const int*>(src)[i];
        };
        copy(sc, a.clusters, a.ncl * int(sizeof(Cluster) / 4));
        copy(sb, a.bounds, a.n * int(sizeof(Bound) / 4));
        copy(ss, a.solids, a.n * int(sizeof(petl_solid) / 4));
        copy(so, a.order, a.n);
        __syncthreads();
    }
    const petl_solid* solids = staged ? ss : a.solids;
    const Bound* bounds = staged ? sb : a.bounds;
    const Cluster* clusters = staged ? sc : a.clusters;
    const int* order = staged ? so : a.order;
    const petl_geom& G = a.G;
    // a warp traces a 4 x 8 (u1 x u0) tile of bins of one view: neighbouring
    // parallel lines, which meet mostly the same solids
    const int tiles_x = (G.N_u0 + 7) / 8, tiles_view = tiles_x * ((G.N_u1 + 3) / 4);
    const long long items = (long long)G.N_v1 * G.N_v0 * tiles_view * 32;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int lane = int(it & 31);
        const long long tile = it >> 5;
        const long long view = tile / tiles_view;
        const int tv = int(tile - view * tiles_view);
        const int iu1 = (tv / tiles_x) * 4 + (lane >> 3), iu0 = (tv % tiles_x) * 8 + (lane & 7);
        if (iu1 >= G.N_u1 || iu0 >= G.N_u0) continue;
        const int iv0 = int(view % G.N_v0), iv1 = int(view / G.N_v0);
        const long long idx = (view * G.N_u1 + iu1) * G.N_u0 + iu0;
        const float v1 = float(iv1) * G.T_v1 + G.v1_0;
        const float v0 = float(iv0) * G.T_v0 + G.v0_0;
        const float u1 = float(iu1) * G.T_u1 + G.u1_0;
        const float u0 = float(iu0) * G.T_u0 + G.u0_0;
        // field of view (the u0 test takes half of T_v0, as the reference's)
        if (fabsf(u1) - 0.5f * G.T_u1 > G.H - G.R * fabsf(v1) ||
            fabsf(u0) - 0.5f * G.T_v0 > G.L + G.R * fabsf(v0)) {
            a.g[idx] = 0.0f;
            continue;
        }
        // direction: the unnormalised direction times its length
        float3 r = make_float3(-(v0 * a.cos_psi + a.sin_psi), -(v0 * a.sin_psi - a.cos_psi), -v1);
        const float len = rsqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
        r = make_float3(r.x / len, r.y / len, r.z / len);
        auto value = [&](float du1, float du0) {
            const float w = u0 + du0;
            const LineSums s =
                line_sums<STOP>(solids, bounds, clusters, a.ncl, order, a.n,
                                make_float3(w * a.cos_psi, w * a.sin_psi, u1 + du1), r);
            return STOP ? (1.0f - expf(-s.fwd)) * (1.0f - expf(-s.bwd)) : s.fwd;
        };
        float out;
        if (a.os <= 1) {
            out = value(0.0f, 0.0f);
        } else {
            const float d1 = G.T_u1 / float(a.os + 1), d0 = G.T_u0 / float(a.os + 1);
            const int rad = (a.os - 1) / 2;
            float acc = 0.0f;
            for (int j = -rad; j <= rad; j++)
                for (int k = -rad; k <= rad; k++) acc += value(float(j) * d1, float(k) * d0);
            out = acc / float(a.os * a.os);
        }
        a.g[idx] = out;
    }
}

// ---------------------------------------------------------------------------
// voxelization
// ---------------------------------------------------------------------------

// One solid as the voxelizer applies it (src/phantom.cpp:141-335).
struct VoxSolid {
    int type;
    float c[3], r[3], val, A[9], clip[3], cone[2];
    int rotated, clipped;
    int lo[3], hi[3];  // voxel index box (x, y, z), clamped
};

__device__ __forceinline__ bool vox_inside(const VoxSolid& s, float x, float y, float z)
{
    auto sq = [](float v) { return __fmul_rn(v, v); };
    bool in = false;
    switch (s.type) {
    case kEllipsoid: in = __fadd_rn(__fadd_rn(sq(x), sq(y)), sq(z)) <= 1.0f; break;
    case kBox: in = fabsf(x) <= 1.0f && fabsf(y) <= 1.0f && fabsf(z) <= 1.0f; break;
    case kCylX: in = fabsf(x) <= 1.0f && __fadd_rn(sq(y), sq(z)) <= 1.0f; break;
    case kCylY: in = fabsf(y) <= 1.0f && __fadd_rn(sq(x), sq(z)) <= 1.0f; break;
    case kCylZ: in = fabsf(z) <= 1.0f && __fadd_rn(sq(x), sq(y)) <= 1.0f; break;
    case kConeX: in = __fadd_rn(sq(y), sq(z)) <= sq(x) && s.cone[0] <= x && x <= s.cone[1]; break;
    case kConeY: in = __fadd_rn(sq(x), sq(z)) <= sq(y) && s.cone[0] <= y && y <= s.cone[1]; break;
    case kConeZ: in = __fadd_rn(sq(x), sq(y)) <= sq(z) && s.cone[0] <= z && z <= s.cone[1]; break;
    default: break;
    }
    if (s.clipped &&
        (__fmul_rn(s.clip[0], x) > 0.0f || __fmul_rn(s.clip[1], y) > 0.0f || __fmul_rn(s.clip[2], z) > 0.0f))
        in = false;
    return in;
}

// Normalised coordinates of a point for the solid, in the reference's float
// operations.
__device__ __forceinline__ bool vox_test(const VoxSolid& s, float x, float y, float z)
{
    const float dx = __fsub_rn(x, s.c[0]), dy = __fsub_rn(y, s.c[1]), dz = __fsub_rn(z, s.c[2]);
    if (!s.rotated) return vox_inside(s, __fdiv_rn(dx, s.r[0]), __fdiv_rn(dy, s.r[1]), __fdiv_rn(dz, s.r[2]));
    float w[3];
    for (int k = 0; k < 3; k++)
        w[k] = __fdiv_rn(
            __fadd_rn(__fadd_rn(__fmul_rn(s.A[3 * k], dx), __fmul_rn(s.A[3 * k + 1], dy)), __fmul_rn(s.A[3 * k + 2], dz)),
            s.r[k]);
    return vox_inside(s, w[0], w[1], w[2]);
}

struct VoxArgs {
    const VoxSolid* solids;
    int n;
    float* f;
    int numX, numY, numZ;
    float T_x, T_z, x_0, y_0, z_0;
    int os;
};

__global__ void k_voxelize(const VoxArgs a)
{
    const long long total = (long long)a.numX * a.numY * a.numZ;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int ix = int(idx % a.numX), iy = int((idx / a.numX) % a.numY), iz = int(idx / ((long long)a.numX * a.numY));
        // voxel centre: i * T + start, float multiply then add (no contraction)
        const float x = __fadd_rn(__fmul_rn(float(ix), a.T_x), a.x_0);
        const float y = __fadd_rn(__fmul_rn(float(iy), a.T_x), a.y_0);
        const float z = __fadd_rn(__fmul_rn(float(iz), a.T_z), a.z_0);
        float v = a.f[idx];
        for (int j = 0; j < a.n; j++) {
            const VoxSolid& s = a.solids[j];
            if (ix < s.lo[0] || ix > s.hi[0] || iy < s.lo[1] || iy > s.hi[1] || iz < s.lo[2] || iz > s.hi[2])
                continue;
            if (a.os == 1) {
                if (vox_test(s, x, y, z)) v = s.val;
                continue;
            }
            // sub-sample k of n at x + T/(n+1) * (k - (n-1)/2), the offset in
            // double; each sub-sample inside moves the value by
            // (val - v) / n^3, accumulated in float through double
            const int os = a.os;
            const double frac = 1.0 / double(float(os * os * os));
            const double half = 0.5 * double(float(os - 1));
            const float step_x = __fdiv_rn(a.T_x, float(os + 1)), step_z = __fdiv_rn(a.T_z, float(os + 1));
            const double dv = __dmul_rn(double(__fsub_rn(s.val, v)), frac);
            float acc = 0.0f;
            for (int kz = 0; kz < os; kz++) {
                const float zs = float(__dadd_rn(double(z), __dmul_rn(double(step_z), double(float(kz)) - half)));
                for (int ky = 0; ky < os; ky++) {
                    const float ys = float(__dadd_rn(double(y), __dmul_rn(double(step_x), double(float(ky)) - half)));
                    for (int kx = 0; kx < os; kx++) {
                        const float xs =
                            float(__dadd_rn(double(x), __dmul_rn(double(step_x), double(float(kx)) - half)));
                        if (vox_test(s, xs, ys, zs)) acc = float(__dadd_rn(double(acc), dv));
                    }
                }
            }
            v = __fadd_rn(acc, v);
        }
        a.f[idx] = v;
    }
}

// The voxelizer's form of a solid (src/phantom.cpp:105-139, 141-232): cones
// rebuilt from the given centre and radii, the first clipping plane as a
// sign mask, the index box from the unrotated (or sqrt(3) max-radius)
// extent, in the reference's host float arithmetic.
VoxSolid vox_form(const petl_solid& s, int numX, int numY, int numZ, float T_x, float T_z, float x_0, float y_0,
                  float z_0)
{
    VoxSolid v{};
    v.type = s.type;
    const bool cone = s.type >= kConeX && s.type <= kConeZ;
    for (int k = 0; k < 3; k++) {
        v.c[k] = cone ? s.given_c[k] : s.centers[k];
        v.r[k] = cone ? s.given_r[k] : s.radii[k];
    }
    v.val = s.val;
    for (int k = 0; k < 9; k++) v.A[k] = s.A[k];
    v.clipped = !cone && s.num_clip > 0;
    for (int k = 0; k < 3; k++) v.clip[k] = -s.clip[0][k];
    const float T[3] = {T_x, T_x, T_z}, o[3] = {x_0, y_0, z_0};
    const int N[3] = {numX, numY, numZ};
    v.rotated = s.A[0] != 1.0f || s.A[4] != 1.0f || s.A[8] != 1.0f;
    float ext[3] = {v.r[0], v.r[1], v.r[2]};
    if (v.rotated || cone) {
        const float rm = float(std::sqrt(3.0) * std::max(v.r[0], std::max(v.r[1], v.r[2])));
        ext[0] = ext[1] = ext[2] = rm;
    }
    for (int k = 0; k < 3; k++) {
        v.lo[k] = int(std::floor((v.c[k] - ext[k] - T[k] - o[k]) / T[k]));
        v.hi[k] = int(std::ceil((v.c[k] + ext[k] + T[k] - o[k]) / T[k]));
    }
    if (cone) {
        const int k = s.type - kConeX;  // axis; the other two radii are the end radii
        const int i0 = k == 0 ? 1 : 0, i1 = k == 2 ? 1 : 2;
        const double l = v.r[k], r1 = v.r[i0], r2 = v.r[i1];
        v.r[i0] = float(std::fabs(r2 - r1) / (2.0 * l));
        v.r[i1] = v.r[i0];
        v.r[k] = 1.0f;
        v.c[k] = float(v.c[k] - l * (r2 + r1) / (r2 - r1));
        v.cone[0] = float(-l + l * (r2 + r1) / (r2 - r1));
        v.cone[1] = float(l + l * (r2 + r1) / (r2 - r1));
    }
    for (int k = 0; k < 3; k++) {
        v.lo[k] = std::max(0, std::min(N[k] - 1, v.lo[k]));
        v.hi[k] = std::max(0, std::min(N[k] - 1, v.hi[k]));
    }
    return v;
}

template <class T>
int upload(const T* host, size_t count, T** dev, cudaStream_t st)
{
    *dev = nullptr;
    if (count == 0) return 0;
    PETL_CUDA(scratch_alloc(reinterpret_cast<void**>(dev), count * sizeof(T), st));
    const cudaError_t e = cudaMemcpyAsync(*dev, host, count * sizeof(T), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(*dev, st);
        *dev = nullptr;
        set_error(std::string("analytic: upload: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace

int voxelize(const petl_solid* solids, int n, float* f, int numX, int numY, int numZ, float T_x, float T_z,
             float x_0, float y_0, float z_0, int oversampling, cudaStream_t st)
{
    PETL_REQUIRE(f && n >= 0 && (n == 0 || solids) && numX > 0 && numY > 0 && numZ > 0 && T_x > 0.f && T_z > 0.f,
                 "voxelize: invalid arguments");
    if (n == 0) return 0;
    std::vector<VoxSolid> vs;
    for (int j = 0; j < n; j++) vs.push_back(vox_form(solids[j], numX, numY, numZ, T_x, T_z, x_0, y_0, z_0));
    VoxSolid* dv = nullptr;
    if (int rc = upload(vs.data(), vs.size(), &dv, st)) return rc;
    VoxArgs a{dv, n, f, numX, numY, numZ, T_x, T_z, x_0, y_0, z_0, std::max(1, std::min(oversampling, 5))};
    const long long total = (long long)numX * numY * numZ;
    const int grid = int(std::min<long long>((total + 255) / 256, 32LL * sm_count()));
    k_voxelize<<<grid, 256, 0, st>>>(a);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(dv, st);
    if (e != cudaSuccess) {
        set_error(std::string("voxelize launch: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

// Padded axis-aligned box around a solid in world coordinates: the solid's
// extents when it is not rotated, else the box of its bounding sphere
// (clipping only removes parts); cones are always tested.
Bound solid_bound(const petl_solid& s)
{
    Bound b{};
    const float* c = s.centers;
    const float* r = s.radii;
    double ext[3] = {std::fabs(double(r[0])), std::fabs(double(r[1])), std::fabs(double(r[2]))};
    if (s.type >= kConeX || s.type < kEllipsoid) {
        b.always = 1;
        return b;
    }
    if (s.rotated) {
        double rad;
        switch (s.type) {
        case kEllipsoid: rad = std::max(ext[0], std::max(ext[1], ext[2])); break;
        case kBox: rad = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]); break;
        case kCylX: rad = std::sqrt(ext[0] * ext[0] + std::pow(std::max(ext[1], ext[2]), 2.0)); break;
        case kCylY: rad = std::sqrt(ext[1] * ext[1] + std::pow(std::max(ext[0], ext[2]), 2.0)); break;
        default: rad = std::sqrt(ext[2] * ext[2] + std::pow(std::max(ext[0], ext[1]), 2.0)); break;
        }
        ext[0] = ext[1] = ext[2] = rad;
    }
    for (int k = 0; k < 3; k++) {
        const double e = ext[k] * (1.0 + 1.0e-4) + 1.0e-3;
        b.lo[k] = float(double(c[k]) - e);
        b.hi[k] = float(double(c[k]) + e);
    }
    return b;
}

// Groups the solids into clusters of up to kClusterSize that lie close
// together: solids always tested in clusters of their own, the others by
// median splits of their box centres along the longest axis.
void make_clusters(const std::vector<Bound>& b, std::vector<Cluster>& cl, std::vector<int>& order)
{
    std::vector<int> boxed, always;
    for (int j = 0; j < int(b.size()); j++) (b[j].always ? always : boxed).push_back(j);
    auto emit = [&](const int* idx, int cnt, bool all) {
        Cluster c{};
        c.first = int(order.size());
        c.count = cnt;
        c.box.always = all ? 1 : 0;
        for (int k = 0; k < 3; k++) {
            c.box.lo[k] = 3.0e38f;
            c.box.hi[k] = -3.0e38f;
        }
        for (int i = 0; i < cnt; i++) {
            order.push_back(idx[i]);
            for (int k = 0; k < 3 && !all; k++) {
                c.box.lo[k] = std::min(c.box.lo[k], b[idx[i]].lo[k]);
                c.box.hi[k] = std::max(c.box.hi[k], b[idx[i]].hi[k]);
            }
        }
        cl.push_back(c);
    };
    for (size_t i = 0; i < always.size(); i += kClusterSize)
        emit(always.data() + i, int(std::min<size_t>(kClusterSize, always.size() - i)), true);
    auto centre = [&](int j, int k) { return 0.5f * (b[j].lo[k] + b[j].hi[k]); };
    std::vector<std::pair<int, int>> todo{{0, int(boxed.size())}};
    while (!todo.empty()) {
        const auto [lo, hi] = todo.back();
        todo.pop_back();
        if (hi - lo <= kClusterSize) {
            if (hi > lo) emit(boxed.data() + lo, hi - lo, false);
            continue;
        }
        float mn[3] = {3.0e38f, 3.0e38f, 3.0e38f}, mx[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
        for (int i = lo; i < hi; i++)
            for (int k = 0; k < 3; k++) {
                mn[k] = std::min(mn[k], centre(boxed[i], k));
                mx[k] = std::max(mx[k], centre(boxed[i], k));
            }
        int ax = 0;
        for (int k = 1; k < 3; k++)
            if (mx[k] - mn[k] > mx[ax] - mn[ax]) ax = k;
        const int mid = (lo + hi) / 2;
        std::nth_element(boxed.begin() + lo, boxed.begin() + mid, boxed.begin() + hi,
                         [&](int x, int y) { return centre(x, ax) < centre(y, ax); });
        todo.push_back({mid, hi});
        todo.push_back({lo, mid});
    }
}

int ray_trace(const petl_geom& G, const petl_solid* solids, int n, float* g, int oversampling, bool stopping,
              cudaStream_t st)
{
    PETL_REQUIRE(g && n >= 0 && (n == 0 || solids) && G.N_v1 > 0 && G.N_v0 > 0 && G.N_u1 > 0 && G.N_u0 > 0,
                 "ray_trace: invalid arguments");
    // oversampling odd, 1..11 (src/analytic_ray_tracing_gpu.cu:871-874)
    int os = std::max(1, std::min(oversampling, 11));
    if (os % 2 == 0) os += 1;
    os = std::max(1, std::min(os, 11));
    petl_solid* ds = nullptr;
    if (int rc = upload(solids, size_t(n), &ds, st)) return rc;
    std::vector<Bound> hb;
    for (int j = 0; j < n; j++) hb.push_back(solid_bound(solids[j]));
    std::vector<Cluster> hc;
    std::vector<int> ho;
    make_clusters(hb, hc, ho);
    Bound* db = nullptr;
    Cluster* dc = nullptr;
    int* dord = nullptr;
    int rc = upload(hb.data(), hb.size(), &db, st);
    if (!rc) rc = upload(hc.data(), hc.size(), &dc, st);
    if (!rc) rc = upload(ho.data(), ho.size(), &dord, st);
    if (rc) {
        for (void* q : {static_cast<void*>(ds), static_cast<void*>(db), static_cast<void*>(dc)})
            if (q) cudaFreeAsync(q, st);
        return rc;
    }
    // the reference's constants: cos/sin of the float psi in float
    RayArgs a{G, ds, db, dc, dord, int(hc.size()), n, g, os, std::cos(G.psi), std::sin(G.psi),
              (long long)G.N_v1 * G.N_v0 * G.N_u1 * G.N_u0};
    const size_t smem =
        n <= kSmemSolids ? hc.size() * sizeof(Cluster) + size_t(n) * (sizeof(petl_solid) + sizeof(Bound) + 4) : 0;
    const int grid = int(std::min<long long>((a.total + kRayThreads - 1) / kRayThreads, 64LL * sm_count()));
    if (stopping)
        k_ray_trace<true><<<grid, kRayThreads, smem, st>>>(a);
    else
        k_ray_trace<false><<<grid, kRayThreads, smem, st>>>(a);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(ds, st);
    cudaFreeAsync(db, st);
    cudaFreeAsync(dc, st);
    cudaFreeAsync(dord, st);
    if (e != cudaSuccess) {
        set_error(std::string("ray_trace launch: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl

extern "C" {

int petl_solid_init(petl_solid* s, int type, const float* c, const float* r, float val, const float* A,
                    const float* clip)
{
    if (!s) return -1;
    *s = petl_solid{};
    s->type = -1;
    if (!c || !r || type < petl::kEllipsoid || type > petl::kConeZ) return -1;
    s->type = type;
    for (int k = 0; k < 3; k++) {
        s->centers[k] = s->given_c[k] = c[k];
        s->radii[k] = s->given_r[k] = r[k];
    }
    if (clip)
        for (int k = 0; k < 3; k++)
            if (clip[k] != 0.0f) {
                s->clip[s->num_clip][k] = -1.0f;
                s->clip[s->num_clip][3] = -clip[k];
                s->num_clip++;
            }
    s->val = val;
    if (A)
        for (int k = 0; k < 9; k++) {
            s->A[k] = A[k];
            const bool diag = k == 0 || k == 4 || k == 8;
            if (std::fabs(double(A[k]) - (diag ? 1.0 : 0.0)) > 1.0e-8) s->rotated = 1;
        }
    if (type >= petl::kConeX) {
        // a cone of unit slope along its axis k, clipped to [clip_cone]
        // (src/phantom.cpp:594-638)
        const int k = type - petl::kConeX, i0 = k == 0 ? 1 : 0, i1 = k == 2 ? 1 : 2;
        const double l = s->radii[k], r1 = s->radii[i0], r2 = s->radii[i1];
        s->radii[i0] = float(std::fabs(r2 - r1) / (2.0 * l));
        s->radii[i1] = s->radii[i0];
        s->radii[k] = 1.0f;
        s->centers[k] = float(s->centers[k] - l * (r2 + r1) / (r2 - r1));
        s->clip_cone[0] = float(-l + l * (r2 + r1) / (r2 - r1));
        s->clip_cone[1] = float(l + l * (r2 + r1) / (r2 - r1));
    }
    return 0;
}

void petl_solids_scale(petl_solid* s, int n, float sx, float sy, float sz)
{
    for (int j = 0; s && j < n; j++) {
        const float f[3] = {sx, sy, sz};
        for (int k = 0; k < 3; k++) {
            s[j].centers[k] *= f[k];
            s[j].radii[k] *= f[k];
        }
        // as the reference: the planes' y and z normals by sy, sz and their
        // offset by sx (src/phantom.cpp:1131-1137)
        for (int i = 0; i < s[j].num_clip; i++) {
            s[j].clip[i][1] *= sy;
            s[j].clip[i][2] *= sz;
            s[j].clip[i][3] *= sx;
        }
    }
}

int petl_voxelize_dev(const petl_solid* solids, int n, float* f, int numX, int numY, int numZ, float voxelWidth,
                      float voxelHeight, float x_0, float y_0, float z_0, int oversampling, void* stream)
{
    return petl::voxelize(solids, n, f, numX, numY, numZ, voxelWidth, voxelHeight, x_0, y_0, z_0, oversampling,
                          petl::as_stream(stream));
}

int petl_ray_trace_dev(const petl_geom* G, const petl_solid* solids, int n, float* g, int oversampling,
                       int stopping_power, void* stream)
{
    PETL_REQUIRE(G != nullptr, "ray_trace: null geometry");
    return petl::ray_trace(*G, solids, n, g, oversampling, stopping_power != 0, petl::as_stream(stream));
}

}  // extern "C"
