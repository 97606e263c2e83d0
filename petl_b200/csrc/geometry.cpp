// Planogram and volume geometry (host side).
//
// Restates planogram::init (reference src/planogram.cpp:143-186),
// parameters::x_0/y_0/z_0 (src/parameters.cpp:271-284) and optimalFFTsize
// (src/vector_ops.cpp:481-505).  The arithmetic keeps the reference's mix of
// float storage and double intermediates so that the sample counts and
// start values come out bit-identical.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cmath>
#include <mutex>
#include <string>

#include "common.cuh"

namespace petl {

namespace {
thread_local std::string g_last_error;
}

std::atomic<unsigned long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

namespace {
std::atomic<long long> g_alloc_countdown{0};  // > 0: the allocation that brings it to 0 fails
std::atomic<long long> g_alloc_count{0};
cudaMemPool_t g_pools[64] = {nullptr};
std::mutex g_pool_mu;
}  // namespace

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st)
{
    g_alloc_count.fetch_add(1, std::memory_order_relaxed);
    if (g_alloc_countdown.load(std::memory_order_relaxed) > 0 &&
        g_alloc_countdown.fetch_sub(1, std::memory_order_relaxed) == 1) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;  // injected (petl_inject_alloc_failure)
    }
    // one library pool per device that keeps freed blocks (release threshold
    // at its maximum): a pool that hands memory back to the system at each
    // synchronisation would map gigabytes of projector scratch anew per call
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        cudaMemPool_t* pools = g_pools;
        if (!pools[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created = nullptr;
            e = cudaMemPoolCreate(&created, &props);
            if (e != cudaSuccess) return e;
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &thr);
            pools[dev] = created;
        }
        pool = pools[dev];
    }
    e = cudaMallocFromPoolAsync(p, bytes, pool, st);
    if (e != cudaSuccess) cudaGetLastError();  // out of memory is not sticky: leave no error behind
    return e;
}

bool geom_valid(const petl_geom* G, std::string* why)
{
    auto bad = [&](const char* m) {
        if (why) *why = m;
        return false;
    };
    if (!G) return bad("null geometry");
    if (G->N_v1 <= 0 || G->N_v0 <= 0 || G->N_u1 <= 0 || G->N_u0 <= 0) return bad("planogram not defined");
    if (!(G->T_v1 > 0.f) || !(G->T_v0 > 0.f) || !(G->T_u1 > 0.f) || !(G->T_u0 > 0.f)) return bad("planogram pitch <= 0");
    if (G->numX <= 0 || G->numY <= 0 || G->numZ <= 0) return bad("volume not defined");
    if (!(G->T_x > 0.f) || !(G->T_z > 0.f)) return bad("voxel size <= 0");
    const double nplan = double(G->N_v1) * G->N_v0 * G->N_u1 * G->N_u0;
    const double nvol = double(G->numX) * G->numY * G->numZ;
    if (nplan > 4.0e10 || nvol > 4.0e10) return bad("array too large");
    return true;
}

}  // namespace petl

extern "C" {

const char* petl_last_error(void) { return petl::g_last_error.c_str(); }

int petl_version(void) { return 100; }

unsigned long long petl_launch_count(void) { return petl::g_launches.load(std::memory_order_relaxed); }

int petl_inject_alloc_failure(long long n)
{
    petl::g_alloc_countdown.store(n > 0 ? n : 0, std::memory_order_relaxed);
    return 0;
}

long long petl_scratch_alloc_count(void) { return petl::g_alloc_count.load(std::memory_order_relaxed); }

long long petl_scratch_in_use(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(petl::g_pool_mu);
        pool = petl::g_pools[dev];
    }
    if (!pool) return 0;
    uint64_t used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) return -1;
    return (long long)used;
}

int petl_optimal_fft_size(int N)
{
    // smallest 2^(n+1)*3^m >= N (src/vector_ops.cpp:481-505), same search
    if (N <= 2) return 2;
    const double c1 = std::log2(double(N) / 2.0) / std::log2(3);
    const double c2 = 1.0 / std::log2(3);
    const double xbar = std::log2(double(N) / 2.0);
    int best = int(std::pow(2, int(std::ceil(xbar)) + 1));
    for (int x = 0; x < int(std::ceil(xbar)); x++) {
        const int y = int(std::ceil(c1 - c2 * double(x)));
        const int v = int(std::pow(2, x + 1) * std::pow(3, y));
        if (v < best && y >= 0) best = v;
    }
    return best;
}

int petl_geom_init(petl_geom* G, float psi_deg, float D, float L, float H, float v_m0, float v_m1, float T)
{
    if (!G) return -1;
    // C-ABI conventions (src/petl_c_interface.cpp:216-219): degrees -> radians,
    // full lengths -> half lengths, computed in double and passed as float
    const double PI = 3.1415926535897932385;
    const float psi = float(psi_deg * PI / 180.0);
    const float R = float(0.5 * D), Lh = float(0.5 * L), Hh = float(0.5 * H);
    if (R <= 0.0 || Lh <= 0.0 || Hh <= 0.0 || v_m0 <= 0.0 || v_m1 < 0.0 || T <= 0.0) {
        petl::set_error("add_planogram: invalid arguments");
        return -1;
    }
    petl_geom g = *G;
    g.psi = psi;
    g.R = R;
    g.L = Lh;
    g.H = Hh;
    g.v_m0 = v_m0;
    g.v_m1 = std::min(Hh / R, v_m1);
    g.T_u0 = T;
    g.T_u1 = T;
    g.T_v0 = g.T_u0 / R;
    g.T_v1 = g.T_u1 / R;
    g.N_u0 = 2 * int((Lh + R * v_m0) / g.T_u0);
    g.N_u1 = 2 * int(Hh / g.T_u1);
    g.N_v0 = 2 * int(v_m0 / g.T_v0) + 1;
    g.N_v1 = 2 * int(g.v_m1 / g.T_v1) + 1;
    g.T_v0 = float(v_m0 * 2.0 / float(g.N_v0));
    g.u0_0 = float(-g.T_u0 * float(g.N_u0 - 1) / 2.0);
    g.u1_0 = float(-g.T_u1 * float(g.N_u1 - 1) / 2.0);
    g.v0_0 = float(-g.T_v0 * float(g.N_v0 - 1) / 2.0);
    g.v1_0 = float(-g.T_v1 * float(g.N_v1 - 1) / 2.0);
    g.cos_psi = float(std::cos(double(psi)));
    g.sin_psi = float(std::sin(double(psi)));
    *G = g;
    return 0;
}

int petl_geom_set_volume(petl_geom* G, int numX, int numY, int numZ, float voxelWidth, float voxelHeight,
                         float offsetX, float offsetY, float offsetZ)
{
    if (!G) return -1;
    if (voxelHeight == 0.0f) voxelHeight = voxelWidth;
    if (!(numX > 0 && numY > 0 && numZ > 0 && voxelWidth > 0.0 && voxelHeight > 0.0)) {
        petl::set_error("set_volume: invalid arguments");
        return -1;
    }
    G->numX = numX;
    G->numY = numY;
    G->numZ = numZ;
    G->T_x = voxelWidth;
    G->T_z = voxelHeight;
    G->x_0 = float((0.0 - 0.5 * (numX - 1)) * voxelWidth + offsetX);
    G->y_0 = float((0.0 - 0.5 * (numY - 1)) * voxelWidth + offsetY);
    G->z_0 = float((0.0 - 0.5 * (numZ - 1)) * voxelHeight + offsetZ);
    return 0;
}

}  // extern "C"
