// Split backprojector with the reference's semantics for any psi.
//
// The reference backprojector (src/projectors.cu:240-377) visits, per voxel
// (x, y, z) and slope v1, the u1 rows of u1 = z + v1 t with
// t = y cos(psi) - x sin(psi), and per view v0 the u0 bins of the voxel's
// projected extent [A, B] (A, B from x cos + y sin + v0 t and the half
// widths).  The depth t does not depend on the view, and the u0 extent does
// not depend on z or v1, so
//   f(x, y, z) = T_x sum_v1 vis sum_u1 w1(v1, t, z, u1) P[v1][u1](x, y),
//   P[v1][u1](x, y) = sum_v0 l_phi(v0, v1) sum_u0 w0(v0, x, y, u0) g[v1][v0][u1][u0],
// the same sums as the reference associated differently (float rounding).
//
// * k_rbp_xy: block = 16 x 16 voxel columns x 32 u1 rows of one slope; per
//   view the rows' u0 window that the tile's extents reach (bounded on the
//   host from the corners of the tile) arrives by cp.async in a ring of
//   three views, column-major (a column's rows contiguous, 16-byte reads);
//   a thread sums two neighbouring voxel columns over the union of their
//   u0 ranges with the reference's box-overlap weights (l_phi folded in).
// * k_rbp_z: thread = voxel column x 8 z rows; per slope the reference's
//   visibility test, u1 box and weights of each row, summed over P.
// P takes N_u1 x numY x numX floats per slope; slopes run in chunks that
// fit the scratch budget.
#include <algorithm>
#include <cmath>
#include <string>

#include "common.cuh"
#include "gsplit.cuh"
#include "projector.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace petl {

namespace {

constexpr int RTX = 16, RTY = 16;                  // voxel columns per k_rbp_xy block
constexpr int RT2 = RTX * RTY / 2;                 // threads per k_rbp_xy block (two columns each)
constexpr int RRB = 32;                            // u1 rows per k_rbp_xy block
constexpr int RRP = RRB + 4;                       // staged floats per column (rows + 16 bytes of padding)
constexpr int RWMAX = 128;                         // staged u0 columns per view at most
constexpr int RSTG = 3;                            // views in flight (cp.async ring)
constexpr int RZB = 8;                             // z rows per k_rbp_z thread (16: 1.1 ms slower at 256x256x128)

struct RxyArgs {
    petl_geom G;
    ViewRange vr;
    int jv1_0;     // first slope of the chunk (index in the range)
    int lgW;       // log2 of the staged u0 columns per view (W <= RWMAX)
    int ntx;       // tiles along x
    int* err;
};

struct RzArgs {
    petl_geom G;
    ViewRange vr;
    int jv1_0, nv1c;  // the chunk's slopes
    int accumulate;
    float scale;
};

// the voxel's view-independent quantities as the reference forms them
__device__ __forceinline__ void voxel_tx(const petl_geom& G, int ix, int iy, float& t, float& xdt)
{
    const float x = fmaf(float(ix), G.T_x, G.x_0);
    const float y = fmaf(float(iy), G.T_x, G.y_0);
    t = fmaf(y, G.cos_psi, -(x * G.sin_psi));
    xdt = fmaf(x, G.cos_psi, y * G.sin_psi);
}

struct ViewU0 {
    float v0, l_phi;
    bool ydom;  // |wy| > |wx|: the extent from the dy half widths
    bool pos;   // the dominant w >= 0 (A from the lower end)
};

__device__ __forceinline__ ViewU0 view_u0(const petl_geom& G, int iv0, float v1)
{
    ViewU0 q;
    q.v0 = fmaf(float(iv0), G.T_v0, G.v0_0);
    const float wy = fmaf(q.v0, G.cos_psi, G.sin_psi);
    const float wx = fmaf(-q.v0, G.sin_psi, G.cos_psi);
    q.l_phi = 1.0f / fmaxf(fabsf(wy), fabsf(wx)) * rsqrtf(1.0f + q.v0 * q.v0 + v1 * v1);
    q.ydom = fabsf(wy) > fabsf(wx);
    q.pos = q.ydom ? wy >= 0.0f : wx >= 0.0f;
    return q;
}

// [A, B]: the voxel's u0 extent in bin units (src/projectors.cu:318-345)
__device__ __forceinline__ void u0_extent(const petl_geom& G, const ViewU0& q, float t, float xdt, float& A, float& B)
{
    const float Tu0_inv = 1.0f / G.T_u0;
    const float sn = G.sin_psi, cs = G.cos_psi;
    const float hx = q.ydom ? 0.5f * G.T_x * sn : 0.5f * G.T_x * cs;   // xdt_dy or xdt_dx
    const float ht = q.ydom ? 0.5f * G.T_x * cs : -0.5f * G.T_x * sn;  // t_dy or t_dx
    const float lo_ = (xdt - hx + q.v0 * (t - ht) - G.u0_0) * Tu0_inv;
    const float hi_ = (xdt + hx + q.v0 * (t + ht) - G.u0_0) * Tu0_inv;
    A = q.pos ? lo_ : hi_;
    B = q.pos ? hi_ : lo_;
}

// 4-byte asynchronous copy global -> shared, zero-filled when !ok
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool ok)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// P[jv1][u1][y][x] for 16 x 16 columns and 32 rows of one slope.  A thread
// takes two neighbouring voxel columns along y (PY) or x, the axis along
// which the u0 extent moves less per voxel, so that their taps share most
// staged columns: it walks the union of their u0 ranges in ascending order
// and applies each staged column (32 rows, 16-byte reads) to both with their
// own weights (predicated off outside a voxel's range, as the reference
// reads no bin outside it).  Grid (tiles, ceil(N_u1 / 32), slopes of the
// chunk); 128 threads; dynamic shared memory: a ring of RSTG views of
// W columns x RRP floats, then the view table.
template <bool PY>
__global__ void __launch_bounds__(RT2, 4) k_rbp_xy(const float* __restrict__ g, float* __restrict__ P,
                                                   const RxyArgs A)
{
    extern __shared__ __align__(16) float rsm[];
    const petl_geom& G = A.G;
    const int tid = threadIdx.x;
    const int tix = blockIdx.x % A.ntx, tiy = blockIdx.x / A.ntx;
    const int x0 = tix * RTX, y0 = tiy * RTY;
    const int xl = min(x0 + RTX, G.numX) - 1, yl = min(y0 + RTY, G.numY) - 1;
    int ix[2], iy[2];
    if (PY) {
        ix[0] = ix[1] = x0 + tid % RTX;
        iy[0] = y0 + 2 * (tid / RTX);
        iy[1] = iy[0] + 1;
    } else {
        ix[0] = x0 + 2 * (tid % (RTX / 2));
        ix[1] = ix[0] + 1;
        iy[0] = iy[1] = y0 + tid / (RTX / 2);
    }
    bool live[2];
    float t[2], xdt[2];
#pragma unroll
    for (int v = 0; v < 2; v++) {
        live[v] = ix[v] < G.numX && iy[v] < G.numY;
        voxel_tx(G, min(ix[v], G.numX - 1), min(iy[v], G.numY - 1), t[v], xdt[v]);
    }
    const int r0 = blockIdx.y * RRB;
    const int jv1 = blockIdx.z;
    const int iv1 = A.vr.iv1_begin + A.jv1_0 + jv1;
    const int lgW = A.lgW, W = 1 << lgW;
    const float v1 = fmaf(float(iv1), G.T_v1, G.v1_0);
    float* ring = rsm;  // [RSTG][W][RRP]
    // per view of the call: first staged column (the smallest first bin over
    // the tile's corners, the extent being affine in x and y, less one of
    // margin) and l_phi
    const int nv0 = A.vr.n_v0(G.N_v0);
    int* s_lo = reinterpret_cast<int*>(rsm + RSTG * W * RRP);
    float* s_lphi = reinterpret_cast<float*>(s_lo + nv0);
    {
        float tc[4], xc[4];
        voxel_tx(G, x0, y0, tc[0], xc[0]);
        voxel_tx(G, xl, y0, tc[1], xc[1]);
        voxel_tx(G, x0, yl, tc[2], xc[2]);
        voxel_tx(G, xl, yl, tc[3], xc[3]);
        for (int k = tid; k < nv0; k += RT2) {
            const ViewU0 q = view_u0(G, A.vr.iv0_first + k * A.vr.iv0_step, v1);
            float m = 3.0e38f;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                float a, b;
                u0_extent(G, q, tc[c], xc[c], a, b);
                m = fminf(m, a);
            }
            s_lo[k] = max(0, int(ceilf(m - 0.5f)) - 1);
            s_lphi[k] = q.l_phi;
        }
    }
    __syncthreads();
    // copies of view k into ring slot k % RSTG: thread e -> row e >> lgW,
    // column e & (W - 1) (coalesced in u0), stored column-major
    auto issue = [&](int k) {
        const int iv0 = A.vr.iv0_first + k * A.vr.iv0_step, lo = s_lo[k];
        float* dst = ring + (k % RSTG) * W * RRP;
        const float* gv = g + (size_t(iv1) * G.N_v0 + iv0) * G.N_u1 * G.N_u0;
        for (int e = tid; e < (RRB << lgW); e += RT2) {
            const int row = e >> lgW, col = e & (W - 1);
            const int iu1 = r0 + row, iu0 = lo + col;
            const bool ok = iu1 < G.N_u1 && iu0 < G.N_u0;
            cp_async4(dst + col * RRP + row, ok ? gv + size_t(iu1) * G.N_u0 + iu0 : g, ok);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < RSTG - 1; k++) {
        if (k < nv0) issue(k);
        else cp_async_commit();
    }

    float acc[2][RRB];
#pragma unroll
    for (int v = 0; v < 2; v++)
#pragma unroll
        for (int r = 0; r < RRB; r++) acc[v][r] = 0.0f;
    for (int k = 0; k < nv0; k++) {
        cp_async_wait<RSTG - 2>();  // this thread's copies of view k landed
        __syncthreads();            // everyone's did; everyone finished reading view k - 1
        if (k + RSTG - 1 < nv0) issue(k + RSTG - 1);  // into the slot of view k - 1
        else cp_async_commit();
        const ViewU0 q = view_u0(G, A.vr.iv0_first + k * A.vr.iv0_step, v1);
        float a[2], b[2];
        int umin[2], umax[2];
#pragma unroll
        for (int v = 0; v < 2; v++) {
            u0_extent(G, q, t[v], xdt[v], a[v], b[v]);
            umin[v] = max(int(ceilf(a[v] - 0.5f)), 0);
            umax[v] = live[v] ? min(int(floorf(b[v] + 0.5f)), G.N_u0 - 1) : -1;
        }
        // the union of the live voxels' ranges
        const int cmin = umax[0] < umin[0] ? umin[1] : umax[1] < umin[1] ? umin[0] : min(umin[0], umin[1]);
        const int cmax = max(umax[0], umax[1]);
        if (cmax < cmin) continue;
        const int lo = s_lo[k];
        if (cmin - lo < 0 || cmax - lo >= W) {  // outside the staged window: the host bound failed
            atomicOr(A.err, kErrLayout);
            continue;
        }
        const float l_phi = s_lphi[k];
        const float* s = ring + (k % RSTG) * W * RRP + (cmin - lo) * RRP;
        for (int c = cmin; c <= cmax; c++, s += RRP) {
            float w[2];
            bool in[2];
#pragma unroll
            for (int v = 0; v < 2; v++) {
                in[v] = c >= umin[v] && c <= umax[v];
                w[v] = l_phi * fmaxf(0.0f, fminf(float(c) + 0.5f, b[v]) - fmaxf(float(c) - 0.5f, a[v]));
            }
            const float4* col = reinterpret_cast<const float4*>(s);
#pragma unroll
            for (int j = 0; j < RRB / 4; j++) {
                const float4 x = col[j];
#pragma unroll
                for (int v = 0; v < 2; v++) {
                    if (!in[v]) continue;
                    acc[v][4 * j] = fmaf(w[v], x.x, acc[v][4 * j]);
                    acc[v][4 * j + 1] = fmaf(w[v], x.y, acc[v][4 * j + 1]);
                    acc[v][4 * j + 2] = fmaf(w[v], x.z, acc[v][4 * j + 2]);
                    acc[v][4 * j + 3] = fmaf(w[v], x.w, acc[v][4 * j + 3]);
                }
            }
        }
    }
    cp_async_wait<0>();
    const size_t plane = size_t(G.numX) * G.numY;
#pragma unroll
    for (int v = 0; v < 2; v++) {
        if (!live[v]) continue;
        float* Pc = P + (size_t(jv1) * G.N_u1 + r0) * plane + size_t(iy[v]) * G.numX + ix[v];
#pragma unroll
        for (int r = 0; r < RRB; r++)
            if (r0 + r < G.N_u1) Pc[size_t(r) * plane] = acc[v][r];
    }
}

// f(x, y, z) (+)= scale T_x sum over the chunk's slopes of the reference's
// u1 taps of P.  Grid (ceil(numX / 32), ceil(numY / 8), ceil(numZ / 8));
// block (32, 8).
__global__ void __launch_bounds__(256) k_rbp_z(const float* __restrict__ P, float* __restrict__ f, const RzArgs A)
{
    const petl_geom& G = A.G;
    const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int iz0 = blockIdx.z * RZB;
    if (ix >= G.numX || iy >= G.numY) return;
    float t, xdt;
    voxel_tx(G, ix, iy, t, xdt);
    const float Tu1_inv = 1.0f / G.T_u1;
    const size_t plane = size_t(G.numX) * G.numY;
    float acc[RZB];
#pragma unroll
    for (int k = 0; k < RZB; k++) acc[k] = 0.0f;
    for (int jv1 = 0; jv1 < A.nv1c; jv1++) {
        const int iv1 = A.vr.iv1_begin + A.jv1_0 + jv1;
        const float v1 = fmaf(float(iv1), G.T_v1, G.v1_0);
        const float* Pv = P + size_t(jv1) * G.N_u1 * plane + size_t(iy) * G.numX + ix;
#pragma unroll
        for (int k = 0; k < RZB; k++) {
            if (iz0 + k >= G.numZ) break;
            const float z = fmaf(float(iz0 + k), G.T_z, G.z_0);
            const float u1 = fmaf(v1, t, z);
            if (!(fabsf(u1) - 0.5f * G.T_u1 <= fmaf(-G.R, fabsf(v1), G.H))) continue;
            const float iu1_mid = (u1 - G.u1_0) * Tu1_inv;
            const float a = iu1_mid - 0.5f * G.T_z * Tu1_inv;
            const float b = iu1_mid + 0.5f * G.T_z * Tu1_inv;
            const int ua = max(int(ceilf(a - 0.5f)), 0);
            const int ub = min(int(floorf(b + 0.5f)), G.N_u1 - 1);
            float sv = 0.0f;
            for (int iu1 = ua; iu1 <= ub; iu1++) {
                const float w1 = fmaxf(0.0f, fminf(float(iu1) + 0.5f, b) - fmaxf(float(iu1) - 0.5f, a));
                if (w1 > 0.0f) sv = fmaf(w1, __ldg(&Pv[size_t(iu1) * plane]), sv);
            }
            acc[k] = fmaf(sv, G.T_x, acc[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < RZB; k++) {
        if (iz0 + k >= G.numZ) break;
        const size_t o = (size_t(iz0 + k) * G.numY + iy) * G.numX + ix;
        const float r = acc[k] * A.scale;
        f[o] = A.accumulate ? f[o] + r : r;
    }
}

}  // namespace

// kNotApplicable when the layout rules fail (the caller then runs the
// general kernel): a u0 extent of three bins or more, a tile window above
// 128 columns, or scratch that cannot be allocated.
int backproject_rsplit(const petl_geom& G, const float* g, float* f, int accumulate, float scale,
                       const ViewRange& vr, cudaStream_t st)
{
    constexpr int kNotApplicable = -2;
    const int n_v0 = vr.n_v0(G.N_v0);
    const int nv1 = vr.iv1_end - vr.iv1_begin;
    if (n_v0 <= 0 || nv1 <= 0) return kNotApplicable;
    // per view: width of the u0 extent (T_x max(|wy|, |wx|) / T_u0) and the
    // spread of its centre over a 16 x 16 tile (15 T_x (|wx| + |wy|) / T_u0)
    // (|wy| is the shift per voxel along y, |wx| along x: a thread's two
    // voxels lie along the axis with the smaller mean shift)
    double wmax = 0, need = 0, sum_wx = 0, sum_wy = 0;
    for (int k = 0; k < n_v0; k++) {
        const double v0 = std::fmaf(float(vr.iv0_first + k * vr.iv0_step), G.T_v0, G.v0_0);
        const double wy = std::fabs(v0 * G.cos_psi + G.sin_psi), wx = std::fabs(-v0 * G.sin_psi + G.cos_psi);
        const double width = double(G.T_x) * std::max(wy, wx) / double(G.T_u0);
        wmax = std::max(wmax, width);
        need = std::max(need, (RTX - 1) * double(G.T_x) * (wx + wy) / double(G.T_u0) + width);
        sum_wx += wx;
        sum_wy += wy;
    }
    // extents of three bins or more (voxels wider than ~3 u0 bins) keep the
    // general kernel
    if (!(wmax < 2.99)) return kNotApplicable;
    const bool pair_y = sum_wy <= sum_wx;
    // + 2 for the bins' rounding, 1 of margin below, 1 of slack; a power of two
    const int wneed = int(std::ceil(need + 4.0));
    int lgW = 4;
    while ((1 << lgW) < wneed) lgW++;
    if ((1 << lgW) > RWMAX) return kNotApplicable;
    const size_t tsmem = size_t(RSTG) * (size_t(1) << lgW) * RRP * 4 + size_t(n_v0) * 8;  // ring + view table
    if (tsmem > 160 * 1024) return kNotApplicable;
    int* err = device_error_ptr();
    if (!err) return kNotApplicable;

    const size_t per_slope = size_t(G.N_u1) * G.numX * G.numY * 4;
    int nc = int(std::max<size_t>(1, std::min<size_t>(size_t(nv1), gsplit_scratch_budget() / per_slope)));
    const int nchunks = (nv1 + nc - 1) / nc;
    nc = (nv1 + nchunks - 1) / nchunks;
    float* P = nullptr;
    if (scratch_alloc(reinterpret_cast<void**>(&P), per_slope * nc, st) != cudaSuccess) {
        cudaGetLastError();
        return kNotApplicable;
    }
    const int ntx = int(ceil_div(G.numX, RTX)), nty = int(ceil_div(G.numY, RTY));
    auto* kxy = pair_y ? k_rbp_xy<true> : k_rbp_xy<false>;
    cudaError_t e = cudaFuncSetAttribute(kxy, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tsmem));
    for (int c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int jv1_0 = c * nc, nvc = std::min(nc, nv1 - jv1_0);
        const RxyArgs XA{G, vr, jv1_0, lgW, ntx, err};
        kxy<<<dim3(unsigned(ntx * nty), ceil_div(G.N_u1, RRB), unsigned(nvc)), RT2, tsmem, st>>>(g, P, XA);
        note_launch();
        const RzArgs ZA{G, vr, jv1_0, nvc, c == 0 ? accumulate : 1, scale};
        k_rbp_z<<<dim3(ceil_div(G.numX, 32), ceil_div(G.numY, 8), ceil_div(G.numZ, RZB)), dim3(32, 8), 0, st>>>(P, f, ZA);
        note_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(P, st);
    if (e != cudaSuccess) {
        set_error(std::string("backproject_rsplit: ") + cudaGetErrorString(e));
        return int(e);
    }
    return 0;
}

}  // namespace petl
