// Shear-warp projector and backprojectors for axis-aligned planograms.
//
// At psi = 0 every ray p + t r with p = (u0, 0, u1), r = (-v0, 1, -v1) is
// y-driven and its parameter on plane y is t = y exactly, so the reference
// footprint (src/projectors.cu:131-185) of voxel (ix, iz) on that plane is
//   w0 = overlap(bin iu0, voxel ix shifted by v0*y),
//   w1 = overlap(bin iu1, voxel iz shifted by v1*y).
// When the voxel pitch equals the bin pitch these overlaps are tent weights
// of a shift that is the same for every voxel of the plane: with
//   s_x(v0, y) = (x_0 + y v0 - u0_0)/T_u0,  dx = floor(-s_x),  phx = -s_x - dx
// (and likewise dz, phz from v1), plane y contributes
//   g[v1][v0][iu1][iu0] += sum_b,a wz_b wx_a f[iu1 + dz + b][y][iu0 + dx + a]
// with wx = (1 - phx, phx), wz = (1 - phz, phz).  The forward kernel applies
// the x shift once per (v0, plane) into shared memory and reuses it for 16
// v1 slopes, so each ray and plane costs two FMAs.  The backward kernels are
// the gather form of the transpose: the z interpolation is summed over v1 in
// registers for several planes at once, then the x shift goes through shared
// memory; every voxel is owned by one CTA, so no atomics are used.
//
// The shifts are evaluated in double from the float geometry (the exact
// arithmetic the reference's float code approximates); ray masks and the
// reference backprojector's voxel-centre test are evaluated with the same
// float expressions as the reference (see projector.cuh) and tabulated.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"

namespace petl {

using shear::Shift;
using shear::Tables;
using shear::TableBuf;

namespace {

// forward tile: 16 v1 x 32 rows x 32 columns, one v0 per CTA
constexpr int FV = 4;    // v1 slopes per thread
constexpr int FK = 16;   // rows per thread
constexpr int FWV = 4;   // warps along v1
constexpr int FWR = 2;   // warps along rows
constexpr int F_THREADS = 32 * FWV * FWR;
constexpr int F_ROWS = FK * FWR;
constexpr int F_V1 = FV * FWV;

// backward tile: NP planes x BK rows per thread, all u0/x columns
constexpr int BNP = 4;
constexpr int BK = 8;

__device__ __forceinline__ float ffv(int i) { return float(i); }

__global__ void k_shear_tables(const petl_geom G, Tables T)
{
    const int n_x = G.N_v0 * G.numY, n_z = G.N_v1 * G.numY, n_s = G.N_v1 * G.N_v0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_x) {
        const int iv0 = i / G.numY, iy = i % G.numY;
        const float v0 = ffma(ffv(iv0), G.T_v0, G.v0_0);
        const float y = ffma(ffv(iy), G.T_x, G.y_0);
        const double m = -((double(G.x_0) + double(y) * double(v0)) - double(G.u0_0)) / double(G.T_u0);
        const double d = floor(m);
        T.xt[i] = Shift{int(d), float(m - d)};
    }
    if (i < n_z) {
        const int iv1 = i / G.numY, iy = i % G.numY;
        const float v1 = ffma(ffv(iv1), G.T_v1, G.v1_0);
        const float y = ffma(ffv(iy), G.T_x, G.y_0);
        const double m = -((double(G.z_0) + double(y) * double(v1)) - double(G.u1_0)) / double(G.T_u1);
        const double d = floor(m);
        T.zt[i] = Shift{int(d), float(m - d)};
        // reference backprojector voxel test: |u1| - T/2 <= H - R|v1|, u1 = fma(v1, y, z)
        int lo = G.numZ, hi = -1;
        for (int iz = 0; iz < G.numZ; iz++) {
            const float z = fmaf(ffv(iz), G.T_z, G.z_0);
            const float u1 = fmaf(v1, y, z);
            if (fabsf(u1) - 0.5f * G.T_u1 <= fmaf(-G.R, fabsf(v1), G.H)) {
                lo = min(lo, iz);
                hi = max(hi, iz);
            }
        }
        T.zvis[i] = make_int2(lo, hi);
    }
    if (i < n_s) {
        const int iv1 = i / G.N_v0, iv0 = i % G.N_v0;
        const float v1 = ffma(ffv(iv1), G.T_v1, G.v1_0);
        const float v0 = ffma(ffv(iv0), G.T_v0, G.v0_0);
        T.S[i] = fmul(G.T_x, __frsqrt_rn(ffma(v0, v0, ffma(v1, v1, 1.0f))));
    }
    if (i < G.N_v0) {
        // the u0 half of ray_visible (it does not depend on v1 or u1)
        int lo = G.N_u0, hi = -1;
        const float v0 = ffma(ffv(i), G.T_v0, G.v0_0);
        for (int iu0 = 0; iu0 < G.N_u0; iu0++) {
            const float u0 = ffma(ffv(iu0), G.T_u0, G.u0_0);
            if (!(fsub(fabsf(u0), fmul(0.5f, G.T_u0)) > ffma(G.R, fabsf(v0), G.L))) {
                lo = min(lo, iu0);
                hi = max(hi, iu0);
            }
        }
        T.ub0[i] = make_int2(lo, hi);
    }
    if (i < G.N_v1) {
        int lo = G.N_u1, hi = -1;
        const float v1 = ffma(ffv(i), G.T_v1, G.v1_0);
        for (int iu1 = 0; iu1 < G.N_u1; iu1++) {
            const float u1 = ffma(ffv(iu1), G.T_u1, G.u1_0);
            if (!(fsub(fabsf(u1), fmul(0.5f, G.T_u1)) > ffma(-G.R, fabsf(v1), G.H))) {
                lo = min(lo, iu1);
                hi = max(hi, iu1);
            }
        }
        T.ub1[i] = make_int2(lo, hi);
    }
}

struct FwdArgs {
    petl_geom G;
    ViewRange vr;
    int n_colblk;
    int maxr;
    Tables T;
};

// ---------------------------------------------------------------------------
// forward projection
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(F_THREADS, 2)
k_fwd_shear(const float* __restrict__ f, float* __restrict__ g, const float* __restrict__ meas, const FwdArgs A)
{
    extern __shared__ float Xs[];  // [2][maxr][32]
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wv = warp % FWV, wr = warp / FWV;
    const int iv0 = A.vr.iv0_first + blockIdx.x * A.vr.iv0_step;
    const int cta_v1_0 = A.vr.iv1_begin + blockIdx.y * F_V1;
    const int cta_v1_1 = min(cta_v1_0 + F_V1, A.vr.iv1_end);
    const int rowblk = blockIdx.z / A.n_colblk, colblk = blockIdx.z % A.n_colblk;
    const int cta_row0 = rowblk * F_ROWS;
    const int col0 = colblk * 32;
    const int col = col0 + lane;
    const int v1w = cta_v1_0 + wv * FV;
    const int row0 = cta_row0 + wr * FK;
    const int NY = G.numY, NX = G.numX, NZ = G.numZ;

    // tile entirely outside the visible bins of every view: store zeros
    const int2 ub0 = A.T.ub0[iv0];
    bool any_row = false;
    for (int v1 = cta_v1_0; v1 < cta_v1_1; v1++) {
        const int2 ub1 = A.T.ub1[v1];
        any_row |= !(cta_row0 > ub1.y || cta_row0 + F_ROWS - 1 < ub1.x);
    }
    const bool live = any_row && !(col0 > ub0.y || col0 + 31 < ub0.x);

    float acc[FV][FK];
#pragma unroll
    for (int a = 0; a < FV; a++)
#pragma unroll
        for (int k = 0; k < FK; k++) acc[a][k] = 0.0f;

    if (live) {
        int par = 0;
        const Shift* xrow = A.T.xt + size_t(iv0) * NY;
        for (int iy = 0; iy < NY; iy++) {
            const Shift xs = xrow[iy];
            const int d_a = A.T.zt[size_t(cta_v1_0) * NY + iy].d;
            const int d_b = A.T.zt[size_t(cta_v1_1 - 1) * NY + iy].d;
            const int dzmin = min(d_a, d_b), dzmax = max(d_a, d_b);
            const int wlo = cta_row0 + dzmin;
            const int nr = F_ROWS + (dzmax - dzmin) + 1;
            const int cx = col0 + xs.d;
            if (cx + 32 < 0 || cx >= NX || wlo + nr - 1 < 0 || wlo >= NZ) continue;  // CTA-uniform
            if (nr > A.maxr) continue;  // cannot happen with the host's bound; never write past the slab
            float* X = Xs + par * A.maxr * 32;
            // stage A: x interpolation of the needed rows of plane iy
            const float wx = xs.w;
            for (int e = tid; e < nr * 32; e += F_THREADS) {
                const int r = e >> 5, c = e & 31;
                const int iz = wlo + r;
                float v = 0.0f;
                if (iz >= 0 && iz < NZ) {
                    const float* fr = f + (size_t(iz) * NY + iy) * NX;
                    const int ix = cx + c;
                    const float a = (ix >= 0 && ix < NX) ? __ldg(fr + ix) : 0.0f;
                    const float b = (ix + 1 >= 0 && ix + 1 < NX) ? __ldg(fr + ix + 1) : 0.0f;
                    v = fmaf(wx, b, (1.0f - wx) * a);
                }
                X[e] = v;
            }
            __syncthreads();
            // stage B: z interpolation into the v1 accumulators
#pragma unroll
            for (int a = 0; a < FV; a++) {
                const int v1 = v1w + a;
                if (v1 < cta_v1_1) {
                    const Shift zs = A.T.zt[size_t(v1) * NY + iy];
                    const float w1 = zs.w, w0 = 1.0f - zs.w;
                    const float* Xr = X + (row0 + zs.d - wlo) * 32 + lane;
                    float xv[FK + 1];
#pragma unroll
                    for (int k = 0; k <= FK; k++) xv[k] = Xr[k * 32];
#pragma unroll
                    for (int k = 0; k < FK; k++) acc[a][k] = fmaf(w1, xv[k + 1], fmaf(w0, xv[k], acc[a][k]));
                }
            }
            par ^= 1;
        }
    }
    // epilogue: scale, ray masks, optional MLEM ratio
    if (col >= G.N_u0) return;
#pragma unroll
    for (int a = 0; a < FV; a++) {
        const int v1 = v1w + a;
        if (v1 >= cta_v1_1) continue;
        const float S = A.T.S[size_t(v1) * G.N_v0 + iv0];
        const int2 ub1 = A.T.ub1[v1];
        const bool colok = col >= ub0.x && col <= ub0.y;
#pragma unroll
        for (int k = 0; k < FK; k++) {
            const int iu1 = row0 + k;
            if (iu1 >= G.N_u1) break;
            const bool vis = colok && iu1 >= ub1.x && iu1 <= ub1.y;
            const float val = vis ? acc[a][k] * S : 0.0f;
            const size_t o = ((size_t(v1) * G.N_v0 + iv0) * G.N_u1 + iu1) * G.N_u0 + col;
            g[o] = meas ? ratio_rule(__ldg(&meas[o]), val) : val;
        }
    }
}

struct BwdArgs {
    petl_geom G;
    ViewRange vr;
    int ncw;  // column warps (ceil(N_u0/32))
    int ng;   // plane groups
    int accumulate;
    float scale;
    Tables T;
};

// ---------------------------------------------------------------------------
// backprojection (gather); ADJ selects the exact transpose of k_fwd_shear
// (bin masks) instead of the reference backprojector (voxel-centre test)
// ---------------------------------------------------------------------------
template <bool ADJ>
__global__ void __launch_bounds__(512, 1)
k_bwd_shear(const float* __restrict__ g, float* __restrict__ f, const BwdArgs A)
{
    extern __shared__ float Zs[];  // [ng*BNP][BK][N_u0]
    const petl_geom& G = A.G;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthreads = blockDim.x;
    const int cw = warp % A.ncw, pg = warp / A.ncw;
    const int NPB = A.ng * BNP;
    const int p0 = blockIdx.x * NPB;   // first plane of the CTA
    const int r0 = blockIdx.y * BK;    // first row (iz) of the CTA
    const int u = cw * 32 + lane;      // planogram column of this thread
    const int NY = G.numY, NX = G.numX, NZ = G.numZ, NU0 = G.N_u0, NU1 = G.N_u1;
    const size_t view_sz = size_t(NU1) * NU0;

    // clear the owned output tile unless accumulating
    if (!A.accumulate) {
        for (int e = tid; e < NPB * BK * NX; e += nthreads) {
            const int p = e / (BK * NX), rem = e - p * BK * NX, k = rem / NX, ix = rem - k * NX;
            const int iy = p0 + p, iz = r0 + k;
            if (iy < NY && iz < NZ) f[(size_t(iz) * NY + iy) * NX + ix] = 0.0f;
        }
    }

    float Z[BNP][BK];
    for (int iv0 = A.vr.iv0_first; iv0 < G.N_v0; iv0 += A.vr.iv0_step) {
#pragma unroll
        for (int p = 0; p < BNP; p++)
#pragma unroll
            for (int k = 0; k < BK; k++) Z[p][k] = 0.0f;
        const int2 ub0 = A.T.ub0[iv0];
        const bool ucol = u < NU0 && (!ADJ || (u >= ub0.x && u <= ub0.y));
        for (int v1 = A.vr.iv1_begin; v1 < A.vr.iv1_end; v1++) {
            const float S = A.T.S[size_t(v1) * G.N_v0 + iv0];
            const float* gv = g + (size_t(v1) * G.N_v0 + iv0) * view_sz;
            int blo = 0, bhi = NU1 - 1;
            if (ADJ) {
                const int2 ub1 = A.T.ub1[v1];
                blo = max(blo, ub1.x);
                bhi = min(bhi, ub1.y);
            }
#pragma unroll
            for (int p = 0; p < BNP; p++) {
                const int iy = p0 + pg * BNP + p;
                if (iy >= NY) break;
                const Shift zs = A.T.zt[size_t(v1) * NY + iy];
                const float w1 = S * zs.w, w0 = S * (1.0f - zs.w);
                const int rb = r0 - zs.d - 1;  // g row of tap 1 for k = 0
                float m[BK];
                if (!ADJ) {
                    const int2 zv = A.T.zvis[size_t(v1) * NY + iy];
#pragma unroll
                    for (int k = 0; k < BK; k++) m[k] = (r0 + k >= zv.x && r0 + k <= zv.y) ? 1.0f : 0.0f;
                }
                float v[BK + 1];
#pragma unroll
                for (int j = 0; j <= BK; j++) {
                    const int row = rb + j;
                    v[j] = (ucol && row >= blo && row <= bhi) ? __ldg(gv + size_t(row) * NU0 + u) : 0.0f;
                }
#pragma unroll
                for (int k = 0; k < BK; k++) {
                    const float t = fmaf(w1, v[k], w0 * v[k + 1]);
                    Z[p][k] = ADJ ? Z[p][k] + t : fmaf(m[k], t, Z[p][k]);
                }
            }
        }
        // x shift of this view into the owned voxels
#pragma unroll
        for (int p = 0; p < BNP; p++)
#pragma unroll
            for (int k = 0; k < BK; k++)
                if (u < NU0) Zs[(size_t(pg * BNP + p) * BK + k) * NU0 + u] = Z[p][k];
        __syncthreads();
        for (int e = tid; e < NPB * BK * NX; e += nthreads) {
            const int p = e / (BK * NX), rem = e - p * BK * NX, k = rem / NX, ix = rem - k * NX;
            const int iy = p0 + p, iz = r0 + k;
            if (iy >= NY || iz >= NZ) continue;
            const Shift xs = A.T.xt[size_t(iv0) * NY + iy];
            const int j0 = ix - xs.d, j1 = j0 - 1;
            const float* zr = Zs + (size_t(p) * BK + k) * NU0;
            const float a = (j0 >= 0 && j0 < NU0) ? zr[j0] : 0.0f;
            const float b = (j1 >= 0 && j1 < NU0) ? zr[j1] : 0.0f;
            const size_t o = (size_t(iz) * NY + iy) * NX + ix;
            f[o] += A.scale * fmaf(xs.w, b, (1.0f - xs.w) * a);
        }
        __syncthreads();
    }
}

}  // namespace

int shear::make_tables(const petl_geom& G, TableBuf& tb, cudaStream_t st)
{
    const size_t nx = size_t(G.N_v0) * G.numY, nz = size_t(G.N_v1) * G.numY, ns = size_t(G.N_v1) * G.N_v0;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_xt = al(nx * sizeof(Shift)), b_zt = al(nz * sizeof(Shift)), b_S = al(ns * 4),
                 b_zv = al(nz * sizeof(int2)), b_u0 = al(G.N_v0 * sizeof(int2)), b_u1 = al(G.N_v1 * sizeof(int2));
    tb.bytes = b_xt + b_zt + b_S + b_zv + b_u0 + b_u1;
    PETL_CUDA(scratch_alloc(&tb.base, tb.bytes, st));
    char* p = static_cast<char*>(tb.base);
    tb.T.xt = reinterpret_cast<Shift*>(p);
    p += b_xt;
    tb.T.zt = reinterpret_cast<Shift*>(p);
    p += b_zt;
    tb.T.S = reinterpret_cast<float*>(p);
    p += b_S;
    tb.T.zvis = reinterpret_cast<int2*>(p);
    p += b_zv;
    tb.T.ub0 = reinterpret_cast<int2*>(p);
    p += b_u0;
    tb.T.ub1 = reinterpret_cast<int2*>(p);
    const size_t n = std::max(std::max(nx, nz), std::max(ns, size_t(std::max(G.N_v0, G.N_v1))));
    k_shear_tables<<<ceil_div(n, 256), 256, 0, st>>>(G, tb.T);
    PETL_LAUNCH_CHECK("shear_tables");
    return 0;
}

namespace {

// ---------------------------------------------------------------------------
// Allocation-free forward projection.
//
// Some callers cannot allocate device memory while they run: a real-time
// acquisition thread that must not block on the allocator, a host program
// that hands the GPU's whole memory to its own pool, or code that must not
// change the device's memory state between two measurements.  For them the
// shear tables of the forward projector live in the fixed array below
// instead of stream-ordered scratch.  The array is a module global: every
// GPU that loads this library holds it (4 MiB) until the process exits, and
// all calls on one device share it, so calls that overlap on the GPU (other
// streams, other host threads) race on its contents.  Each call rewrites the
// whole table region it uses before reading it, so nothing needs clearing
// between calls.
constexpr size_t kNoAllocTableBytes = size_t(4) << 20;
static __device__ __align__(256) unsigned char g_noalloc_tables[kNoAllocTableBytes];

size_t tables_size(const petl_geom& G)
{
    const size_t nx = size_t(G.N_v0) * G.numY, nz = size_t(G.N_v1) * G.numY, ns = size_t(G.N_v1) * G.N_v0;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    return al(nx * sizeof(Shift)) + al(nz * sizeof(Shift)) + al(ns * 4) + al(nz * sizeof(int2)) +
           al(G.N_v0 * sizeof(int2)) + al(G.N_v1 * sizeof(int2));
}

// Device address of the fixed table array, looked up once per device with
// that device current (the host-side name of the array is not a device
// address).
int noalloc_table_base(void** out)
{
    static std::mutex mu;
    static void* base[64] = {nullptr};
    int dev = 0;
    PETL_CUDA(cudaGetDevice(&dev));
    PETL_REQUIRE(dev >= 0 && dev < 64, "no-alloc projection: device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!base[dev]) {
        void* p = nullptr;
        PETL_CUDA(cudaGetSymbolAddress(&p, g_noalloc_tables));
        base[dev] = p;
    }
    *out = base[dev];
    return 0;
}

}  // namespace

bool shear_eligible(const petl_geom& G)
{
    if (!(G.cos_psi == 1.0f && G.sin_psi == 0.0f)) return false;
    if (!(G.T_x == G.T_u0 && G.T_z == G.T_u1)) return false;
    // every view y-driven: |v0| < 1 at both ends of the slope range
    const float va = std::fmaf(0.0f, G.T_v0, G.v0_0), vb = std::fmaf(float(G.N_v0 - 1), G.T_v0, G.v0_0);
    if (!(std::fabs(va) < 1.0f && std::fabs(vb) < 1.0f)) return false;
    if (G.N_u0 > 32 * 16 || G.numX > 4096) return false;
    return true;
}

int shear::project_with(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                        const Tables& T, cudaStream_t st)
{
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return 0;
    if (dispatch_mode() != 2) {
        const int rc = shear::project_tma(G, f, g, vr, meas, T, st);
        if (rc != shear::kNotApplicable) {
            note_path(2);
            return rc;
        }
    }
    note_path(1);
    // rows of the staged slab: 32 output rows + the spread of 16 slopes + 1
    const double ymax = std::max(std::fabs(double(G.y_0)), std::fabs(double(G.y_0) + (G.numY - 1) * double(G.T_x)));
    const int spread = int(std::ceil(double(F_V1) * double(G.T_v1) * ymax / double(G.T_z))) + 4;
    FwdArgs A{};
    A.G = G;
    A.vr = vr;
    A.n_colblk = int(ceil_div(G.N_u0, 32));
    A.maxr = F_ROWS + spread + 1;
    A.T = T;
    const size_t smem = size_t(2) * A.maxr * 32 * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(k_fwd_shear, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) {
        dim3 grid(unsigned(n_v0), ceil_div(nv1, F_V1), unsigned(A.n_colblk) * ceil_div(G.N_u1, F_ROWS));
        k_fwd_shear<<<grid, F_THREADS, smem, st>>>(f, g, meas, A);
        note_launch();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error(std::string("project_shear: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

size_t shear::table_bytes(const petl_geom& G) { return tables_size(G); }

int launch_project_shear(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                         cudaStream_t st)
{
    if (vr.n_v0(G.N_v0) <= 0 || vr.iv1_end <= vr.iv1_begin) return 0;
    TableBuf tb;
    int rc = shear::make_tables(G, tb, st);
    if (rc) return rc;
    rc = shear::project_with(G, f, g, vr, meas, tb.T, st);
    cudaFreeAsync(tb.base, st);
    return rc;
}

int shear::project_chunked(const petl_geom& G, const float* f, float* g, int chunk_cap, const ChunkHook& hook,
                           cudaStream_t st)
{
    if (dispatch_mode() != 0 || !shear_eligible(G)) return kNotApplicable;
    TableBuf tb;
    int rc = shear::make_tables(G, tb, st);
    if (rc) return rc;
    const ViewRange vr{0, G.N_v1, 0, 1};
    rc = shear::project_split(G, f, g, vr, nullptr, tb.T, st, chunk_cap, &hook);
    cudaFreeAsync(tb.base, st);
    if (rc == 0) note_path(2);
    return rc;
}

int shear::backproject_chunked(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                               int chunk_cap, const ChunkHook& hook, cudaStream_t st)
{
    if (dispatch_mode() != 0 || !shear_eligible(G)) return kNotApplicable;
    TableBuf tb;
    int rc = shear::make_tables(G, tb, st);
    if (rc) return rc;
    const ViewRange vr{0, G.N_v1, 0, 1};
    rc = shear::backproject_split(G, g, f, mode, accumulate, scale, vr, tb.T, st, chunk_cap, &hook);
    cudaFreeAsync(tb.base, st);
    if (rc == 0) note_path(2);
    return rc;
}

int shear::backproject_with(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                            const ViewRange& vr, const Tables& T, cudaStream_t st)
{
    if (dispatch_mode() != 2) {
        const int rc = shear::backproject_tma(G, g, f, mode, accumulate, scale, vr, T, st);
        if (rc != shear::kNotApplicable) {
            note_path(2);
            return rc;
        }
    }
    note_path(1);
    BwdArgs A{};
    A.G = G;
    A.vr = vr;
    A.ncw = int(ceil_div(G.N_u0, 32));
    A.ng = std::max(1, std::min(2, 16 / A.ncw));
    A.accumulate = accumulate;
    A.scale = scale;
    A.T = T;
    const int threads = A.ncw * 32 * A.ng;
    const size_t smem = size_t(A.ng) * BNP * BK * G.N_u0 * sizeof(float);
    cudaError_t e = cudaSuccess;
    dim3 grid(ceil_div(G.numY, A.ng * BNP), ceil_div(G.numZ, BK));
    if (mode == PETL_BP_ADJOINT) {
        e = cudaFuncSetAttribute(k_bwd_shear<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) k_bwd_shear<true><<<grid, threads, smem, st>>>(g, f, A);
    } else {
        e = cudaFuncSetAttribute(k_bwd_shear<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) k_bwd_shear<false><<<grid, threads, smem, st>>>(g, f, A);
    }
    note_launch();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("backproject_shear: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

int launch_backproject_shear(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                             const ViewRange& vr, cudaStream_t st)
{
    TableBuf tb;
    int rc = shear::make_tables(G, tb, st);
    if (rc) return rc;
    rc = shear::backproject_with(G, g, f, mode, accumulate, scale, vr, tb.T, st);
    cudaFreeAsync(tb.base, st);
    return rc;
}

}  // namespace petl

using namespace petl;

extern "C" int petl_project_noalloc_dev(const petl_geom* G, const float* f, float* g, void* stream)
{
    clear_error();
    std::string why;
    PETL_REQUIRE(G && f && g && geom_valid(G, &why), "project_noalloc: invalid arguments " + why);
    cudaStream_t st = as_stream(stream);
    const ViewRange vr{0, G->N_v1, 0, 1};
    // geometries outside the shear kernels' domain (or a forced general
    // dispatch) use the general kernel, which needs no scratch memory at all
    if (dispatch_mode() == 1 || !shear_eligible(*G)) {
        note_path(0);
        return launch_project_general(*G, f, g, vr, nullptr, st);
    }
    const size_t need = tables_size(*G);
    if (need > kNoAllocTableBytes) {
        set_error("project_noalloc: this geometry needs " + std::to_string(need) +
                  " bytes of table scratch; the allocation-free entry point holds at most " +
                  std::to_string(kNoAllocTableBytes) + " bytes");
        return -1;
    }
    void* base = nullptr;
    int rc = noalloc_table_base(&base);
    if (rc) return rc;
    // same table layout as the allocating path, placed in the fixed array
    const size_t nx = size_t(G->N_v0) * G->numY, nz = size_t(G->N_v1) * G->numY, ns = size_t(G->N_v1) * G->N_v0;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    Tables T{};
    char* p = static_cast<char*>(base);
    T.xt = reinterpret_cast<Shift*>(p);
    p += al(nx * sizeof(Shift));
    T.zt = reinterpret_cast<Shift*>(p);
    p += al(nz * sizeof(Shift));
    T.S = reinterpret_cast<float*>(p);
    p += al(ns * 4);
    T.zvis = reinterpret_cast<int2*>(p);
    p += al(nz * sizeof(int2));
    T.ub0 = reinterpret_cast<int2*>(p);
    p += al(G->N_v0 * sizeof(int2));
    T.ub1 = reinterpret_cast<int2*>(p);
    const size_t n = std::max(std::max(nx, nz), std::max(ns, size_t(std::max(G->N_v0, G->N_v1))));
    k_shear_tables<<<ceil_div(n, 256), 256, 0, st>>>(*G, T);
    PETL_LAUNCH_CHECK("shear_tables (no-alloc)");
    const double ymax =
        std::max(std::fabs(double(G->y_0)), std::fabs(double(G->y_0) + (G->numY - 1) * double(G->T_x)));
    const int spread = int(std::ceil(double(F_V1) * double(G->T_v1) * ymax / double(G->T_z))) + 4;
    FwdArgs A{};
    A.G = *G;
    A.vr = vr;
    A.n_colblk = int(ceil_div(G->N_u0, 32));
    A.maxr = F_ROWS + spread + 1;
    A.T = T;
    const size_t smem = size_t(2) * A.maxr * 32 * sizeof(float);
    PETL_CUDA(cudaFuncSetAttribute(k_fwd_shear, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 grid(unsigned(G->N_v0), ceil_div(G->N_v1, F_V1), unsigned(A.n_colblk) * ceil_div(G->N_u1, F_ROWS));
    k_fwd_shear<<<grid, F_THREADS, smem, st>>>(f, g, nullptr, A);
    PETL_LAUNCH_CHECK("project_noalloc");
    note_path(1);
    return 0;
}
