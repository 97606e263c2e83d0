// List-mode binning of coincidences into planograms on the device.
//
// The reference reads coincidences from a file into per-planogram queues and
// flushes each queue on the host with OpenMP over v1 slices
// (src/binning.cpp:558-790).  Here the host only parses the file into
// batches of event pairs (pinned staging, two batches in flight); one thread
// per event and planogram maps the pair to planogram coordinates
// (planogram::is_within_acceptable_angle / get_u_coords,
// src/planogram.cpp:113-141), applies the chest-wall shift
// (src/binning.cpp:630-645) and deposits the event with atomic adds: nearest
// bin, or bilinear weights in (u1, u0) computed in double as the reference's
// flush_queue computes them.  Float arithmetic uses rounding-pinned
// intrinsics so that the coordinates round as the reference's host code
// rounds them; only the order of the additions into one bin differs (exact
// for unit weights in nearest mode, last-bit differences in linear mode).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace petl {

namespace {

// int(x + 0.5) with the addition in double, as the reference writes it
__device__ __forceinline__ int round_half_up_trunc(float x) { return __double2int_rz(__dadd_rn(double(x), 0.5)); }

__global__ void k_bin_events(const petl_geom G, const float* __restrict__ blue, const float* __restrict__ pink,
                             long long n, float* __restrict__ g, int linear, int chest_wall)
{
    const size_t proj = size_t(G.N_u1) * G.N_u0, obl = size_t(G.N_v0) * proj;
    const float cs = G.cos_psi, sn = G.sin_psi;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const float bx = blue[3 * e], by = blue[3 * e + 1], bz = blue[3 * e + 2];
        const float r0 = fsub(bx, pink[3 * e]), r1 = fsub(by, pink[3 * e + 1]), r2 = fsub(bz, pink[3 * e + 2]);
        // is_within_acceptable_angle
        const float c = fadd(fmul(-sn, r0), fmul(cs, r1));
        if (c == 0.0f) continue;
        const float v0 = __fdiv_rn(-fadd(fmul(cs, r0), fmul(sn, r1)), c);
        if (fabsf(v0) > G.v_m0) continue;
        const float v1 = __fdiv_rn(-r2, c);
        if (fabsf(v1) > G.v_m1) continue;
        // get_u_coords of the blue end, then the chest-wall origin
        const float t = fsub(fmul(by, cs), fmul(bx, sn));
        float u1 = fadd(bz, fmul(v1, t));
        const float u0 = fadd(fadd(fmul(bx, cs), fmul(by, sn)), fmul(v0, t));
        if (chest_wall) u1 = fsub(u1, G.H);
        // flush_queue: slope and view of the event
        const int iv1 = round_half_up_trunc(__fdiv_rn(fsub(v1, G.v1_0), G.T_v1));
        if (iv1 < 0 || iv1 >= G.N_v1) continue;
        const int iv0 = round_half_up_trunc(__fdiv_rn(fsub(v0, G.v0_0), G.T_v0));
        if (iv0 < 0 || iv0 >= G.N_v0) continue;
        float* P = g + size_t(iv1) * obl + size_t(iv0) * proj;
        const float fu1 = __fdiv_rn(fsub(u1, G.u1_0), G.T_u1), fu0 = __fdiv_rn(fsub(u0, G.u0_0), G.T_u0);
        if (!linear) {
            const int a = round_half_up_trunc(fu1), b = round_half_up_trunc(fu0);
            if (a >= 0 && a < G.N_u1 && b >= 0 && b < G.N_u0) atomicAdd(P + size_t(a) * G.N_u0 + b, 1.0f);
            continue;
        }
        int lo1, hi1, lo0, hi0;
        float d1, d0;
        if (fu1 <= 0.0f) {
            lo1 = hi1 = 0;
            d1 = 0.0f;
        } else if (fu1 >= float(G.N_u1 - 1)) {
            lo1 = hi1 = G.N_u1 - 1;
            d1 = 0.0f;
        } else {
            lo1 = int(fu1);
            hi1 = lo1 + 1;
            d1 = fsub(fu1, float(lo1));
        }
        if (fu0 <= 0.0f) {
            lo0 = hi0 = 0;
            d0 = 0.0f;
        } else if (fu0 >= float(G.N_u0 - 1)) {
            lo0 = hi0 = G.N_u0 - 1;
            d0 = 0.0f;
        } else {
            lo0 = int(fu0);
            hi0 = lo0 + 1;
            d0 = fsub(fu0, float(lo0));
        }
        // weights in double, (1 - d1)(1 - d0) w with w = 1 (every event has weight 1)
        const double e1 = __dsub_rn(1.0, double(d1)), e0 = __dsub_rn(1.0, double(d0));
        atomicAdd(P + lo1 * G.N_u0 + lo0, float(__dmul_rn(e1, e0)));
        atomicAdd(P + hi1 * G.N_u0 + lo0, float(__dmul_rn(double(d1), e0)));
        atomicAdd(P + lo1 * G.N_u0 + hi0, float(__dmul_rn(e1, double(d0))));
        atomicAdd(P + hi1 * G.N_u0 + hi0, float(__dmul_rn(double(d1), double(d0))));
    }
}

}  // namespace

int launch_bin_events(const petl_geom& G, const float* blue, const float* pink, long long n, float* g, int linear,
                      int chest_wall, cudaStream_t st)
{
    if (n <= 0) return 0;
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)sm_count() * 16);
    k_bin_events<<<unsigned(blocks), 256, 0, st>>>(G, blue, pink, n, g, linear, chest_wall);
    PETL_LAUNCH_CHECK("bin_events");
    return 0;
}

// ---------------------------------------------------------------------------
// List-mode files (the reference's two formats, src/binning.cpp:67-151 and
// 558-660), parsed on the host in batches.
// ---------------------------------------------------------------------------
namespace {

struct Reader {
    FILE* fh = nullptr;
    bool lst = false;
    long long remaining = -1;  // coincidences announced by the header (binary format)
    std::vector<unsigned char> buf;
    size_t pos = 0, len = 0;
    bool eof = false;

    bool fill(size_t need)
    {
        if (len - pos >= need) return true;
        std::memmove(buf.data(), buf.data() + pos, len - pos);
        len -= pos;
        pos = 0;
        while (!eof && len < need) {
            const size_t got = std::fread(buf.data() + len, 1, buf.size() - len, fh);
            if (got == 0) eof = true;
            len += got;
        }
        return len - pos >= need;
    }
    template <class T>
    T take()
    {
        T v;
        std::memcpy(&v, buf.data() + pos, sizeof(T));
        pos += sizeof(T);
        return v;
    }
    // next coincidence; false at the end of the data
    bool next(float* b, float* p)
    {
        if (lst) {
            if (!fill(48)) return false;
            std::memcpy(b, buf.data() + pos, 12);
            std::memcpy(p, buf.data() + pos + 24, 12);
            pos += 48;
            return true;
        }
        if (remaining == 0) return false;
        for (int side = 0; side < 2; side++) {
            if (!fill(18)) return false;
            const short nint = take<short>();
            float* q = side == 0 ? b : p;
            std::memcpy(q, buf.data() + pos, 12);
            pos += 16;  // position and energy
            for (int k = 1; k < nint; k++) {  // further interactions: skipped
                if (!fill(18)) return false;
                pos += 18;
            }
        }
        remaining--;
        return true;
    }
};

bool ends_with(const std::string& s, const char* suf)
{
    const size_t n = std::strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

}  // namespace

// Bins the coincidences of a list-mode file into device planograms dg[i]
// (zeroed here) of the planograms `plans`.  The host parses batches of up to
// kBatch events into pinned staging while the device bins the previous one.
int bin_file(const std::vector<petl_geom>& plans, const std::vector<float*>& dg, const char* path, int linear,
             int chest_wall, cudaStream_t st, long long* binned_events)
{
    constexpr long long kBatch = 1 << 20;
    Reader rd;
    rd.fh = std::fopen(path, "rb");
    PETL_REQUIRE(rd.fh != nullptr, std::string("bin: cannot open list-mode file ") + path);
    rd.lst = ends_with(path, ".lst");
    rd.buf.resize(size_t(8) << 20);
    if (!rd.lst) {
        if (!rd.fill(8)) {
            std::fclose(rd.fh);
            set_error("bin: list-mode file too short for its header");
            return -1;
        }
        rd.remaining = rd.take<long long>();
    }
    for (size_t i = 0; i < plans.size(); i++) {
        const size_t n = size_t(plans[i].N_v1) * plans[i].N_v0 * plans[i].N_u1 * plans[i].N_u0;
        PETL_CUDA(cudaMemsetAsync(dg[i], 0, n * 4, st));
    }
    float* host[2] = {nullptr, nullptr};
    float* dev[2] = {nullptr, nullptr};
    cudaEvent_t used[2] = {nullptr, nullptr};
    int rc = 0;
    auto fail = [&](cudaError_t e, const char* what) {
        set_error(std::string("bin: ") + what + ": " + cudaGetErrorString(e));
        rc = int(e);
    };
    for (int s = 0; s < 2 && !rc; s++) {
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&host[s]), size_t(kBatch) * 24, cudaHostAllocDefault);
        if (e == cudaSuccess) e = scratch_alloc(reinterpret_cast<void**>(&dev[s]), size_t(kBatch) * 24, st);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&used[s], cudaEventDisableTiming);
        if (e != cudaSuccess) fail(e, "staging");
    }
    long long total = 0;
    for (int s = 0; !rc; s ^= 1) {
        // the copy that last read this staging buffer must be done
        if (cudaEventSynchronize(used[s]) != cudaSuccess) {
            fail(cudaGetLastError(), "sync");
            break;
        }
        float* hb = host[s];
        float* hp = host[s] + 3 * kBatch;
        long long m = 0;
        while (m < kBatch && rd.next(hb + 3 * m, hp + 3 * m)) m++;
        if (m == 0) break;
        cudaError_t e = cudaMemcpyAsync(dev[s], hb, size_t(m) * 12, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dev[s] + 3 * kBatch, hp, size_t(m) * 12, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(used[s], st);
        if (e != cudaSuccess) {
            fail(e, "copy");
            break;
        }
        for (size_t i = 0; i < plans.size() && !rc; i++)
            rc = launch_bin_events(plans[i], dev[s], dev[s] + 3 * kBatch, m, dg[i], linear, chest_wall, st);
        total += m;
        if (m < kBatch) break;
    }
    std::fclose(rd.fh);
    cudaStreamSynchronize(st);
    for (int s = 0; s < 2; s++) {
        if (host[s]) cudaFreeHost(host[s]);
        if (dev[s]) cudaFreeAsync(dev[s], st);
        if (used[s]) cudaEventDestroy(used[s]);
    }
    if (binned_events) *binned_events = total;
    return rc;
}

}  // namespace petl

using namespace petl;

extern "C" int petl_bin_events_dev(const petl_geom* G, const float* blue, const float* pink, long long n, float* g,
                                   int linear, int chest_wall, void* stream)
{
    clear_error();
    PETL_REQUIRE(G && (n == 0 || (blue && pink && g)) && n >= 0, "bin_events: invalid arguments");
    PETL_REQUIRE(G->N_v1 > 0 && G->N_v0 > 0 && G->N_u1 > 0 && G->N_u0 > 0 && G->T_v1 > 0 && G->T_v0 > 0 &&
                     G->T_u1 > 0 && G->T_u0 > 0,
                 "bin_events: the planogram is not defined");
    return launch_bin_events(*G, blue, pink, n, g, linear, chest_wall, as_stream(stream));
}
