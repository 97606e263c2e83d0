// The reference-compatible C ABI (include/petl.h): model registry, geometry
// setters/getters and host-pointer entry points.
//
// Restates src/petl_c_interface.cpp (whole file), src/list_of_models.cpp:37-46
// (get() appends a model when the list is empty and wraps the index modulo
// the list size), src/parameters.cpp (volume / planogram bookkeeping,
// set_default_volume at 205-248) and src/petl.cpp:205-385 (per-planogram
// orchestration, FBP through PFDR when N_v1 > 1).  Differences by design:
//  * one stream-ordered device pool replaces cudaMalloc/cudaFree per call;
//  * projections stream their output back slab by slab (a copy stream runs
//    behind the compute stream), backprojections stream their input in the
//    same way and accumulate over slabs, so host<->device transfers overlap
//    the kernels;
//  * the elementwise helpers (multiply/divide/rdivide/reciprocal/
//    inner_product) act on host arrays exactly as the reference's OpenMP
//    dataCube code does; their device-resident twins are in petl_device.h.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/petl.h"
#include "../../include/petl_device.h"

extern "C" {
int petl_project_range_dev(const petl_geom* G, const float* f, float* g, int iv1_begin, int iv1_end, int iv0_first,
                           int iv0_step, void* stream);
int petl_backproject_range_dev(const petl_geom* G, const float* g, float* f, int mode, int accumulate, float scale,
                               int iv1_begin, int iv1_end, int iv0_first, int iv0_step, void* stream);
int petl_gaussian_filter_dev(float* f, int N1, int N2, int N3, float FWHM, int numDims, void* stream);
}

namespace petl {
int fbp(const petl_geom& G, const float* g, float* f, int accumulate, cudaStream_t st, float* host_rebinned_out);
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st);
int bin_file(const std::vector<petl_geom>& plans, const std::vector<float*>& dg, const char* path, int linear,
             int chest_wall, cudaStream_t st, long long* binned_events);
int solid_angle(const petl_geom& G, float* g, bool inverse, int iv1_b, int iv1_e, cudaStream_t st);
int apply_corrections(const petl_geom& G, float* g, const float* r, float rel, int iv1_b, int iv1_e,
                      cudaStream_t st);
namespace shear {
struct ChunkHook {
    void (*fn)(void* ctx, int vi0, int nvc) = nullptr;
    void* ctx = nullptr;
};
constexpr int kNotApplicable = -2;
int project_chunked(const petl_geom& G, const float* f, float* g, int chunk_cap, const ChunkHook& hook,
                    cudaStream_t st);
int backproject_chunked(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                        int chunk_cap, const ChunkHook& hook, cudaStream_t st);
}  // namespace shear
}  // namespace petl

namespace {

const char* kVersion = "1.0";

struct Params {
    std::vector<petl_geom> plans;  // planogram fields only
    int numX = 0, numY = 0, numZ = 0;
    float voxelWidth = 0.f, voxelHeight = 0.f;
    float offsetX = 0.f, offsetY = 0.f, offsetZ = 0.f;

    void clearAll()
    {
        numX = numY = numZ = 0;
        voxelWidth = voxelHeight = 0.f;
        offsetX = offsetY = offsetZ = 0.f;
        plans.clear();
    }
    bool volumeDefined(bool print = true) const
    {
        if (numX <= 0 || numY <= 0 || numZ <= 0 || voxelWidth <= 0.0 || voxelHeight <= 0.0) {
            if (print) {
                printf("numZ = %d voxelHeight = %f\n", numZ, voxelHeight);
                printf("Error: volume voxel sizes and number of data elements must be positive\n");
            }
            return false;
        }
        return true;
    }
    static bool planDefined(const petl_geom& p)
    {
        return p.R > 0.0 && p.L > 0.0 && p.H > 0.0 && p.v_m0 > 0.0 && p.v_m1 >= 0.0 && p.T_u0 > 0.0 &&
               p.T_u1 > 0.0 && p.T_v0 > 0.0 && p.T_v1 > 0.0 && p.N_u0 > 0 && p.N_u1 > 0 && p.N_v0 > 0 && p.N_v1 > 0;
    }
    bool geometryDefined() const
    {
        if (plans.empty()) return false;
        for (const auto& p : plans)
            if (!planDefined(p)) return false;
        return true;
    }
    bool allDefined() const { return geometryDefined() && volumeDefined(); }
    petl_geom full(size_t i) const
    {
        petl_geom G = plans[i];
        petl_geom_set_volume(&G, numX, numY, numZ, voxelWidth, voxelHeight, offsetX, offsetY, offsetZ);
        return G;
    }
    size_t volElems() const { return size_t(numX) * numY * numZ; }
};

struct Model {
    Params params;
    std::vector<petl_solid> phantom, modules;  // analytic solids (src/petl.h:140-141)
};

std::mutex g_mu;
std::vector<std::unique_ptr<Model>> g_models;
int g_which = 0;

Model* tomo()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_models.empty()) g_models.emplace_back(new Model);
    return g_models[size_t(g_which) % g_models.size()].get();
}

// --- per-device streams for the host-pointer entry points -------------------
struct DevCtx {
    cudaStream_t compute = nullptr, copy = nullptr;
    bool ok = false;
};

DevCtx* dev_ctx()
{
    static std::mutex mu;
    static DevCtx ctx[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    DevCtx& c = ctx[dev];
    if (!c.ok) {
        if (cudaStreamCreateWithFlags(&c.compute, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        if (cudaStreamCreateWithFlags(&c.copy, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        // keep freed blocks in the stream-ordered pool between calls
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        c.ok = true;
    }
    return &c;
}

bool report(const char* what, int rc)
{
    if (rc != 0) {
        fprintf(stderr, "%s failed: %s\n", what, petl_last_error());
        return false;
    }
    return true;
}

// The kernels' bounded waits record a give-up (and a failed host-side layout
// bound) in the device error word instead of hanging; a call whose kernels
// did so has incomplete outputs and fails.  Read after the call's final
// synchronisation (reading clears the word).
bool device_ok(const char* what)
{
    const int flag = petl_device_error_flag();
    if (flag > 0) {
        fprintf(stderr, "%s failed: device error word %d (1: a bounded wait gave up, 2: a layout bound)\n", what,
                flag);
        return false;
    }
    return true;
}

bool cuda_ok(const char* what, cudaError_t e)
{
    if (e != cudaSuccess) {
        fprintf(stderr, "%s failed: %s\n", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Host <-> device copies of caller arrays.  Pinned (page-locked) host memory
// is copied directly and asynchronously.  Pageable memory -- a plain numpy
// array, what the reference binding passes -- moves through a ring of four
// 32 MB pinned buffers per device: the DMA of one buffer overlaps the
// multi-threaded host copy of another (the driver's own pageable copies run
// at 11-20 GB/s on this class of machine; page-locking the caller's array for
// one call costs more than it saves).  Staged copies return once the host
// side is done: device to host, the data is in the caller's array; host to
// device, the caller's array has been read and the DMAs are queued on the
// stream.
// ---------------------------------------------------------------------------
constexpr int kRingSlots = 4;
constexpr size_t kRingBytes = size_t(32) << 20;

struct Ring {
    std::mutex mu;
    char* buf[kRingSlots] = {};
    cudaEvent_t ev[kRingSlots] = {};
    int next = 0;
    bool ready = false;
};

Ring* ring_for_device()
{
    static Ring rings[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    return &rings[dev];
}

bool ring_init(Ring& r)
{
    if (r.ready) return true;
    for (int k = 0; k < kRingSlots; k++) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&r.buf[k]), kRingBytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming) != cudaSuccess)
            return false;
    }
    r.ready = true;
    return true;
}

bool host_pinned(const void* p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer: pageable
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

// Many host copies at once: one parallel region over blocks of up to 1 MB of
// all of them.
struct CopyJob {
    char* dst;
    const char* src;
    size_t bytes;
};

void par_memcpy(const std::vector<CopyJob>& jobs)
{
    const size_t block = size_t(1) << 20;
    std::vector<CopyJob> blocks;
    for (const CopyJob& j : jobs)
        for (size_t o = 0; o < j.bytes; o += block) blocks.push_back({j.dst + o, j.src + o, std::min(block, j.bytes - o)});
    const long long nb = (long long)blocks.size();
#pragma omp parallel for schedule(static)
    for (long long b = 0; b < nb; b++) std::memcpy(blocks[size_t(b)].dst, blocks[size_t(b)].src, blocks[size_t(b)].bytes);
}

// A strided block: rows of `width` bytes, `height` of them, at pitches
// hpitch (host) and dpitch (device).
struct Block {
    char* host;
    char* dev;
    size_t hpitch, dpitch, width, height;
};

// Pieces of the block that fit in ring slots, in order: (row, offset, bytes).
template <class F>
void for_pieces(const Block& b, F f)
{
    for (size_t y = 0; y < b.height; y++)
        for (size_t o = 0; o < b.width; o += kRingBytes) f(y, o, std::min(kRingBytes, b.width - o));
}

cudaError_t staged_d2h(const Block& b, cudaStream_t st)
{
    Ring* r = ring_for_device();
    if (!r) return cudaErrorNoDevice;
    std::lock_guard<std::mutex> lk(r->mu);
    if (!ring_init(*r)) return cudaErrorMemoryAllocation;
    struct Piece {
        char* host;
        size_t off, bytes;
    };
    std::vector<Piece> batch[kRingSlots];
    std::vector<int> queue;  // slots with copies in flight, oldest first
    size_t fill = 0;
    int slot = r->next;
    auto consume = [&](int k) -> cudaError_t {
        const cudaError_t e = cudaEventSynchronize(r->ev[k]);
        if (e != cudaSuccess) return e;
        std::vector<CopyJob> jobs;
        for (const Piece& pc : batch[k]) jobs.push_back({pc.host, r->buf[k] + pc.off, pc.bytes});
        par_memcpy(jobs);
        batch[k].clear();
        return cudaSuccess;
    };
    auto close = [&]() -> cudaError_t {
        if (batch[slot].empty()) return cudaSuccess;
        cudaError_t e = cudaEventRecord(r->ev[slot], st);
        if (e != cudaSuccess) return e;
        queue.push_back(slot);
        slot = (slot + 1) % kRingSlots;
        fill = 0;
        if (int(queue.size()) == kRingSlots) {  // the next slot is the oldest: empty it
            e = consume(queue.front());
            queue.erase(queue.begin());
        }
        return e;
    };
    cudaError_t e = cudaSuccess;
    for_pieces(b, [&](size_t y, size_t o, size_t n) {
        if (e != cudaSuccess) return;
        if (fill + n > kRingBytes) e = close();
        if (e != cudaSuccess) return;
        // the slot's last user may be an upload on another stream whose DMA
        // out of the slot is still queued: this stream waits for it
        if (fill == 0) e = cudaStreamWaitEvent(st, r->ev[slot], 0);
        if (e != cudaSuccess) return;
        e = cudaMemcpyAsync(r->buf[slot] + fill, b.dev + y * b.dpitch + o, n, cudaMemcpyDeviceToHost, st);
        batch[slot].push_back({b.host + y * b.hpitch + o, fill, n});
        fill += n;
    });
    if (e == cudaSuccess) e = close();
    for (int k : queue) {
        const cudaError_t e2 = consume(k);
        if (e == cudaSuccess) e = e2;
    }
    r->next = slot;
    return e;
}

cudaError_t staged_h2d(const Block& b, cudaStream_t st)
{
    Ring* r = ring_for_device();
    if (!r) return cudaErrorNoDevice;
    std::lock_guard<std::mutex> lk(r->mu);
    if (!ring_init(*r)) return cudaErrorMemoryAllocation;
    struct Piece {
        const char* host;
        char* dev;
        size_t off, bytes;
    };
    std::vector<Piece> batch;
    size_t fill = 0;
    int slot = r->next;
    cudaError_t e = cudaSuccess;
    auto flush = [&]() {
        if (batch.empty() || e != cudaSuccess) return;
        // the slot's previous copies have left it
        e = cudaEventSynchronize(r->ev[slot]);
        std::vector<CopyJob> jobs;
        for (const Piece& pc : batch) jobs.push_back({r->buf[slot] + pc.off, pc.host, pc.bytes});
        par_memcpy(jobs);
        for (const Piece& pc : batch)
            if (e == cudaSuccess) e = cudaMemcpyAsync(pc.dev, r->buf[slot] + pc.off, pc.bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(r->ev[slot], st);
        batch.clear();
        fill = 0;
        slot = (slot + 1) % kRingSlots;
    };
    for_pieces(b, [&](size_t y, size_t o, size_t n) {
        if (fill + n > kRingBytes) flush();
        batch.push_back({b.host + y * b.hpitch + o, b.dev + y * b.dpitch + o, fill, n});
        fill += n;
    });
    flush();
    r->next = slot;
    return e;
}

// cudaMemcpy2DAsync / cudaMemcpyAsync between a caller's host array and the
// device, staged when the host array is pageable.
cudaError_t copy_d2h_2d(void* host, size_t hpitch, const void* dev, size_t dpitch, size_t width, size_t height,
                        cudaStream_t st)
{
    if (host_pinned(host))
        return cudaMemcpy2DAsync(host, hpitch, dev, dpitch, width, height, cudaMemcpyDeviceToHost, st);
    return staged_d2h(Block{static_cast<char*>(host), const_cast<char*>(static_cast<const char*>(dev)), hpitch,
                            dpitch, width, height},
                      st);
}
cudaError_t copy_h2d_2d(void* dev, size_t dpitch, const void* host, size_t hpitch, size_t width, size_t height,
                        cudaStream_t st)
{
    if (host_pinned(host))
        return cudaMemcpy2DAsync(dev, dpitch, host, hpitch, width, height, cudaMemcpyHostToDevice, st);
    return staged_h2d(Block{const_cast<char*>(static_cast<const char*>(host)), static_cast<char*>(dev), hpitch,
                            dpitch, width, height},
                      st);
}
cudaError_t copy_d2h(void* host, const void* dev, size_t bytes, cudaStream_t st)
{
    return copy_d2h_2d(host, bytes, dev, bytes, bytes, 1, st);
}
cudaError_t copy_h2d(void* dev, const void* host, size_t bytes, cudaStream_t st)
{
    return copy_h2d_2d(dev, bytes, host, bytes, bytes, 1, st);
}

// Scoped device allocation from the stream-ordered pool.
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t err = cudaSuccess;  // of the last alloc()
    bool alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        err = petl::scratch_alloc(&p, bytes ? bytes : 4, s);
        if (err != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();  // an allocation failure is not sticky: clear it
        }
        return err == cudaSuccess;
    }
    ~DevBuf()
    {
        if (p) cudaFreeAsync(p, st);
    }
    float* f() const { return static_cast<float*>(p); }
};

// Views per pipeline stage of the split projectors: each stage's planogram
// views move across PCIe while the next stage computes.
constexpr int kChunkViews = 16;

// Copies views [vi0, vi0 + nvc) of every slope of a planogram between host
// and device (a strided block: one row of views per slope), on `copy`,
// ordered after the work enqueued so far on `compute` (device to host) or
// followed by a wait of `compute` (host to device).
// A pageable destination is copied one chunk late (staged copies block the
// host until the data is in place, so the chunk after it must already be
// queued on the device); flush() copies what is left.
struct ViewCopy {
    petl_geom G;
    float* host;
    float* dev;
    cudaStream_t compute, copy;
    bool to_host;
    bool ok = true;
    bool pinned = true;
    std::vector<std::pair<int, int>> pending;  // chunks (vi0, nvc) not yet copied to a pageable host array
    void d2h(int vi0, int nvc)
    {
        const size_t vb = size_t(G.N_u1) * G.N_u0 * 4, pitch = vb * G.N_v0, off = (size_t(vi0) * vb) / 4;
        ok = ok && cuda_ok("project D2H", copy_d2h_2d(host + off, pitch, dev + off, pitch, vb * nvc, G.N_v1, copy));
    }
    void flush()
    {
        for (const auto& pc : pending) d2h(pc.first, pc.second);
        pending.clear();
    }
    static void run(void* ctx, int vi0, int nvc)
    {
        ViewCopy& c = *static_cast<ViewCopy*>(ctx);
        const size_t vb = size_t(c.G.N_u1) * c.G.N_u0 * 4, pitch = vb * c.G.N_v0, off = (size_t(vi0) * vb) / 4;
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (c.to_host) {
            // the previous chunk first: the copy stream already follows its
            // compute, and not yet this chunk's
            if (!c.pinned) c.flush();
            cudaEventRecord(ev, c.compute);
            cudaStreamWaitEvent(c.copy, ev, 0);
            if (c.pinned)
                c.d2h(vi0, nvc);
            else
                c.pending.push_back({vi0, nvc});
        } else {
            c.ok = c.ok && cuda_ok("backproject H2D", copy_h2d_2d(c.dev + off, pitch, c.host + off, pitch, vb * nvc,
                                                                  c.G.N_v1, c.copy));
            cudaEventRecord(ev, c.copy);
            cudaStreamWaitEvent(c.compute, ev, 0);
        }
        cudaEventDestroy(ev);
    }
};

// v1 slices per pipeline stage of the other projectors: a multiple of 16
// (the slopes one forward CTA covers, so no stage launches part-empty
// tiles) moving up to ~256 MB
int slab_step(const petl_geom& G)
{
    const double slab_bytes = double(G.N_v0) * G.N_u1 * G.N_u0 * 4.0;
    const int blocks = int(std::max(1.0, std::floor(256.0e6 / std::max(16.0 * slab_bytes, 1.0))));
    return std::min(16 * blocks, G.N_v1);
}

// ---------------------------------------------------------------------------
// host elementwise rules (src/data_cube.cpp:97-166), OpenMP as the reference
// ---------------------------------------------------------------------------
enum BinOp { MULT, DIV, RDIV };

bool binop(float* x, float* y, size_t n, BinOp op)
{
    const long long N = (long long)n;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; i++) {
        switch (op) {
        case MULT: x[i] *= y[i]; break;
        case DIV: x[i] = (y[i] == 0.0f) ? 0.0f : x[i] / y[i]; break;
        case RDIV: x[i] = (x[i] == 0.0f) ? 0.0f : y[i] / x[i]; break;
        }
    }
    return true;
}

float inner(const float* x, const float* y, const float* w, size_t slab, size_t nslab)
{
    // per-slab double sums, then a double total (src/data_cube.cpp:360-394)
    std::vector<double> sums(nslab, 0.0);
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)nslab; s++) {
        double acc = 0.0;
        const size_t o = size_t(s) * slab;
        for (size_t k = 0; k < slab; k++)
            acc += w ? double(x[o + k] * y[o + k] * w[o + k]) : double(x[o + k] * y[o + k]);
        sums[s] = acc;
    }
    double total = 0.0;
    for (double v : sums) total += v;
    return float(total);
}

// Runs op on each slab of v1 rows of every planogram: the slab's data (and
// response) go up on the copy stream, op runs on the compute stream once they
// have arrived, and the slab's result comes back on the compute stream, so
// uploads of later slabs overlap the downloads of earlier ones.
template <class Op>
bool stream_planograms(const Params& P, float** g, float** r, const char* what, Op op)
{
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok(what, cudaErrorNoDevice);
    bool ok = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom& G = P.plans[i];
        const size_t slab = size_t(G.N_v0) * G.N_u1 * G.N_u0, n = slab * G.N_v1;
        DevBuf dg, dr;
        if (!dg.alloc(n * 4, c->compute) || (r && !dr.alloc(n * 4, c->compute)))
            return cuda_ok(what, dg.err != cudaSuccess ? dg.err : dr.err);
        // the copy stream may only write the buffers once they exist
        cudaEvent_t ready;
        cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
        cudaEventRecord(ready, c->compute);
        cudaStreamWaitEvent(c->copy, ready, 0);
        cudaEventDestroy(ready);
        const int step = slab_step(G);
        for (int b = 0; b < G.N_v1 && ok; b += step) {
            const int e = std::min(G.N_v1, b + step);
            const size_t off = size_t(b) * slab, bytes = size_t(e - b) * slab * 4;
            ok = cuda_ok(what, copy_h2d(dg.f() + off, g[i] + off, bytes, c->copy));
            if (r) ok = ok && cuda_ok(what, copy_h2d(dr.f() + off, r[i] + off, bytes, c->copy));
            cudaEvent_t ev;
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            cudaEventRecord(ev, c->copy);
            cudaStreamWaitEvent(c->compute, ev, 0);
            cudaEventDestroy(ev);
            ok = ok && report(what, op(G, dg.f(), r ? dr.f() : nullptr, b, e, c->compute));
            ok = ok && cuda_ok(what, copy_d2h(g[i] + off, dg.f() + off, bytes, c->compute));
        }
    }
    ok = cuda_ok(what, cudaStreamSynchronize(c->copy)) && ok;
    ok = cuda_ok(what, cudaStreamSynchronize(c->compute)) && ok;
    return ok;
}


}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// registry
// ---------------------------------------------------------------------------
bool set_model(int i)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_which = i;
    return true;
}

int create_new_model(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_models.emplace_back(new Model);
    g_which = int(g_models.size()) - 1;
    return g_which;
}

void about(void)
{
    printf("***********************************************************\n");
    printf("       Planogram Emission Tomography Library (PETL)\n");
    printf("                 version %s (B200 build)\n", kVersion);
    printf("***********************************************************\n");
}

bool copy_parameters(int param_id)
{
    Model* cur = tomo();
    std::lock_guard<std::mutex> lk(g_mu);
    if (0 <= param_id && param_id < int(g_models.size())) {
        if (g_which != param_id) cur->params = g_models[param_id]->params;
        return true;
    }
    return false;
}

void clearAll(void) { tomo()->params.clearAll(); }

void print_parameters(void)
{
    const Params& P = tomo()->params;
    auto x0 = [&](int n, float w, float o) { return float((0.0 - 0.5 * (n - 1)) * w + o); };
    printf("\n======== PET Volume ========\n");
    printf("number of voxels (x, y, z): %d x %d x %d\n", P.numX, P.numY, P.numZ);
    printf("voxel size: %f mm x %f mm x %f mm\n", P.voxelWidth, P.voxelWidth, P.voxelHeight);
    if (P.offsetX != 0.0 || P.offsetY != 0.0 || P.offsetZ != 0.0)
        printf("volume offset: %f mm, %f mm, %f mm\n", P.offsetX, P.offsetY, P.offsetZ);
    printf("FOV: [%f, %f] x [%f, %f] x [%f, %f]\n", x0(P.numX, P.voxelWidth, P.offsetX) - 0.5 * P.voxelWidth,
           (P.numX - 1) * P.voxelWidth + x0(P.numX, P.voxelWidth, P.offsetX) + 0.5 * P.voxelWidth,
           x0(P.numY, P.voxelWidth, P.offsetY) - 0.5 * P.voxelWidth,
           (P.numY - 1) * P.voxelWidth + x0(P.numY, P.voxelWidth, P.offsetY) + 0.5 * P.voxelWidth,
           x0(P.numZ, P.voxelHeight, P.offsetZ) - 0.5 * P.voxelHeight,
           (P.numZ - 1) * P.voxelHeight + x0(P.numZ, P.voxelHeight, P.offsetZ) + 0.5 * P.voxelHeight);
    printf("\n======== PET Geometry ========\n");
    for (size_t i = 0; i < P.plans.size(); i++) {
        const petl_geom& p = P.plans[i];
        printf("Planogram %d\n", int(i));
        printf("  angle = %f deg\n", p.psi * 180.0 / 3.1415926535897932385);
        printf("  number of samples: %d x %d x %d x %d\n", p.N_v1, p.N_v0, p.N_u1, p.N_u0);
        printf("  detector size: %f mm x %f mm\n", p.T_u1, p.T_u0);
        printf("  full detector length: %f mm\n", 2.0 * p.L);
        printf("  full detector height: %f mm\n", 2.0 * p.H);
        printf("  distance between panels: %f mm\n", 2.0 * p.R);
    }
    int ndev = 0;
    cudaGetDeviceCount(&ndev);
    printf("\n======== Settings ========\nGPUs: %d\n%d CPU threads\n\n", ndev, omp_get_num_procs());
}

bool volume_defined(void) { return tomo()->params.volumeDefined(); }
bool geometry_defined(void) { return tomo()->params.geometryDefined(); }

int get_numX(void) { return tomo()->params.numX; }
bool set_numX(int N) { if (N > 0) { tomo()->params.numX = N; return true; } return false; }
int get_numY(void) { return tomo()->params.numY; }
bool set_numY(int N) { if (N > 0) { tomo()->params.numY = N; return true; } return false; }
int get_numZ(void) { return tomo()->params.numZ; }
bool set_numZ(int N) { if (N > 0) { tomo()->params.numZ = N; return true; } return false; }
float get_voxelWidth(void) { return tomo()->params.voxelWidth; }
bool set_voxelWidth(float w) { if (w > 0.0) { tomo()->params.voxelWidth = w; return true; } return false; }
float get_voxelHeight(void) { return tomo()->params.voxelHeight; }
bool set_voxelHeight(float h) { if (h > 0.0) { tomo()->params.voxelHeight = h; return true; } return false; }
// the reference accepts only positive offsets in these setters
// (src/petl_c_interface.cpp:154-195); set_volume accepts any offset
float get_offsetX(void) { return tomo()->params.offsetX; }
bool set_offsetX(float v) { if (v > 0.0) { tomo()->params.offsetX = v; return true; } return false; }
float get_offsetY(void) { return tomo()->params.offsetY; }
bool set_offsetY(float v) { if (v > 0.0) { tomo()->params.offsetY = v; return true; } return false; }
float get_offsetZ(void) { return tomo()->params.offsetZ; }
bool set_offsetZ(float v) { if (v > 0.0) { tomo()->params.offsetZ = v; return true; } return false; }

int get_numPlanograms(void) { return int(tomo()->params.plans.size()); }

bool get_planogramSize(int which, int* shape)
{
    const Params& P = tomo()->params;
    if (!P.geometryDefined() || which < 0 || which >= int(P.plans.size()) || shape == nullptr) return false;
    const petl_geom& p = P.plans[which];
    shape[0] = p.N_v1;
    shape[1] = p.N_v0;
    shape[2] = p.N_u1;
    shape[3] = p.N_u0;
    return true;
}

bool add_planogram(float psi, float R, float L, float H, float v_m0, float v_m1, float T)
{
    petl_geom g{};
    if (petl_geom_init(&g, psi, R, L, H, v_m0, v_m1, T) != 0) return false;
    tomo()->params.plans.push_back(g);
    return true;
}

int petl_model_geometry(int which, petl_geom* out)
{
    const Params& P = tomo()->params;
    if (!out || which < 0 || which >= int(P.plans.size())) return -1;
    *out = P.volumeDefined(false) ? P.full(size_t(which)) : P.plans[size_t(which)];
    return 0;
}

int petl_copy_to_host(void* host, const void* dev, long long bytes, void* stream)
{
    if (!host || !dev || bytes < 0) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = copy_d2h(host, dev, size_t(bytes), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? 0 : int(e);
}

int petl_copy_to_device(void* dev, const void* host, long long bytes, void* stream)
{
    if (!host || !dev || bytes < 0) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = copy_h2d(dev, host, size_t(bytes), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? 0 : int(e);
}

int petl_model_solids(int modules, petl_solid* out, int capacity)
{
    const Model* m = tomo();
    const std::vector<petl_solid>& v = modules ? m->modules : m->phantom;
    for (int i = 0; out && i < capacity && i < int(v.size()); i++) out[i] = v[size_t(i)];
    return int(v.size());
}

bool remove_planogram(int which)
{
    auto& v = tomo()->params.plans;
    if (which >= 0 && which < int(v.size())) {
        v.erase(v.begin() + which);
        return true;
    }
    return false;
}

bool keep_only_planogram(int which)
{
    auto& v = tomo()->params.plans;
    if (which >= 0 && which < int(v.size())) {
        const petl_geom keep = v[which];
        v.assign(1, keep);
        return true;
    }
    return false;
}

bool set_default_volume(float scale)
{
    // parameters::set_default_volume (src/parameters.cpp:205-248)
    Params& P = tomo()->params;
    if (!P.geometryDefined()) return false;
    P.offsetX = P.offsetY = P.offsetZ = 0.0f;
    float X = 0, Y = 0, Z = 0;
    for (size_t i = 0; i < P.plans.size(); i++) {
        const petl_geom& p = P.plans[i];
        const float W = p.L, Hh = p.R;
        const float Xn = float(std::fabs(W * std::cos(double(p.psi))) + std::fabs(Hh * std::sin(double(p.psi))));
        const float Yn = float(std::fabs(W * std::sin(double(p.psi))) + std::fabs(Hh * std::cos(double(p.psi))));
        if (i == 0) {
            P.voxelWidth = p.T_u0;
            P.voxelHeight = p.T_u1;
            Z = p.H;
            X = Xn;
            Y = Yn;
        } else {
            P.voxelWidth = std::min(P.voxelWidth, p.T_u0);
            P.voxelHeight = std::min(P.voxelHeight, p.T_u1);
            Z = std::min(Z, p.H);
            X = std::min(X, Xn);
            Y = std::min(Y, Yn);
        }
    }
    P.voxelWidth *= scale;
    P.voxelHeight *= scale;
    P.numZ = 2 * int(Z / P.voxelHeight);
    P.numY = 2 * int(Y / P.voxelWidth);
    P.numX = 2 * int(X / P.voxelWidth);
    return true;
}

bool set_volume(int numX, int numY, int numZ, float voxelWidth, float voxelHeight, float offsetX, float offsetY,
                float offsetZ)
{
    if (numX > 0 && numY > 0 && numZ > 0 && voxelWidth > 0.0 && voxelHeight > 0.0) {
        Params& P = tomo()->params;
        P.numX = numX;
        P.numY = numY;
        P.numZ = numZ;
        P.voxelWidth = voxelWidth;
        P.voxelHeight = voxelHeight;
        P.offsetX = offsetX;
        P.offsetY = offsetY;
        P.offsetZ = offsetZ;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// list-mode binning
// ---------------------------------------------------------------------------
bool bin(float** g, char* file_name)
{
    // PETL::bin (src/petl.cpp:65-79): the planograms are overwritten with the
    // file's coincidences, binned with the reference's defaults (bilinear in
    // (u1, u0), z from the chest wall, mm)
    const Params P = tomo()->params;
    if (g == nullptr || file_name == nullptr || file_name[0] == 0 || !P.geometryDefined()) return false;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("bin", cudaErrorNoDevice);
    std::vector<std::unique_ptr<DevBuf>> bufs;
    std::vector<float*> dg;
    for (const petl_geom& G : P.plans) {
        bufs.emplace_back(new DevBuf);
        const size_t n = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0;
        if (!bufs.back()->alloc(n * 4, c->compute)) return cuda_ok("bin alloc", bufs.back()->err);
        dg.push_back(bufs.back()->f());
    }
    long long events = 0;
    bool ok = report("bin", petl::bin_file(P.plans, dg, file_name, 1, 1, c->compute, &events));
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom& G = P.plans[i];
        const size_t n = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0;
        ok = cuda_ok("bin D2H", copy_d2h(g[i], dg[i], n * 4, c->compute));
    }
    ok = cuda_ok("bin sync", cudaStreamSynchronize(c->compute)) && ok;
    return ok;
}
// the reference's scatter simulation validates its inputs and computes
// nothing (src/petl.cpp:194-202)
bool simulate_scatter(float** g, float* mu) { return g != nullptr && mu != nullptr && tomo()->params.allDefined(); }

// ---------------------------------------------------------------------------
// analytic phantoms and detector modules (src/petl_c_interface.cpp:271-301,
// src/petl.cpp:81-152)
// ---------------------------------------------------------------------------
static bool add_solid(std::vector<petl_solid>& list, int type, float* c, float* r, float val, float* A, float* clip)
{
    petl_solid sd;
    if (petl_solid_init(&sd, type, c, r, val, A, clip) != 0) return false;
    list.push_back(sd);
    return true;
}
bool add_object(int type, float* c, float* r, float val, float* A, float* clip)
{
    return add_solid(tomo()->phantom, type, c, r, val, A, clip);
}
bool add_module(int type, float* c, float* r, float val, float* A, float* clip)
{
    return add_solid(tomo()->modules, type, c, r, val, A, clip);
}
bool clear_phantom(void)
{
    tomo()->phantom.clear();
    return true;
}
bool clear_modules(void)
{
    tomo()->modules.clear();
    return true;
}
bool scale_phantom(float sx, float sy, float sz)
{
    Model* m = tomo();
    petl_solids_scale(m->phantom.data(), int(m->phantom.size()), sx, sy, sz);
    return true;
}

// phantom::voxelize into the host volume f (values outside every solid are
// kept), on the GPU
bool voxelize(float* f, int oversampling)
{
    Model* m = tomo();
    const Params P = m->params;
    if (f == nullptr || !P.volumeDefined()) return false;
    const std::vector<petl_solid> solids = m->phantom;
    if (solids.empty()) return true;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("voxelize", cudaErrorNoDevice);
    petl_geom Gv{};
    petl_geom_set_volume(&Gv, P.numX, P.numY, P.numZ, P.voxelWidth, P.voxelHeight, P.offsetX, P.offsetY,
                         P.offsetZ);
    const size_t n = P.volElems();
    DevBuf df;
    if (!df.alloc(n * 4, c->compute)) return cuda_ok("voxelize alloc", df.err);
    bool ok = cuda_ok("voxelize H2D", copy_h2d(df.f(), f, n * 4, c->compute));
    ok = ok && report("voxelize", petl_voxelize_dev(solids.data(), int(solids.size()), df.f(), P.numX, P.numY,
                                                    P.numZ, P.voxelWidth, P.voxelHeight, Gv.x_0, Gv.y_0, Gv.z_0,
                                                    oversampling, c->compute));
    ok = ok && cuda_ok("voxelize D2H", copy_d2h(f, df.f(), n * 4, c->compute));
    return cuda_ok("voxelize sync", cudaStreamSynchronize(c->compute)) && ok;
}

static bool trace_planograms(float** g, int oversampling, bool stopping, const char* what)
{
    Model* m = tomo();
    const Params P = m->params;
    if (g == nullptr || !P.geometryDefined()) return false;
    const std::vector<petl_solid> solids = stopping ? m->modules : m->phantom;
    if (stopping && solids.empty()) {
        // no module model: unit stopping power (src/petl.cpp:139-147)
        for (size_t i = 0; i < P.plans.size(); i++) {
            const petl_geom& G = P.plans[i];
            std::fill(g[i], g[i] + size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0, 1.0f);
        }
        return true;
    }
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok(what, cudaErrorNoDevice);
    bool ok = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom& G = P.plans[i];
        const size_t n = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0;
        DevBuf dg;
        if (!dg.alloc(n * 4, c->compute)) return cuda_ok(what, dg.err);
        ok = report(what, petl_ray_trace_dev(&G, solids.data(), int(solids.size()), dg.f(), oversampling,
                                             stopping ? 1 : 0, c->compute));
        ok = ok && cuda_ok(what, copy_d2h(g[i], dg.f(), n * 4, c->compute));
    }
    return cuda_ok(what, cudaStreamSynchronize(c->compute)) && ok;
}
bool ray_trace(float** g, int oversampling) { return trace_planograms(g, oversampling, false, "ray_trace"); }
bool stopping_power(float** g, int oversampling)
{
    return trace_planograms(g, oversampling, true, "stopping_power");
}

// PETL::set_solid_angle_correction (src/petl.cpp:154-162)
bool set_solid_angle_correction(float** g, bool do_inverse)
{
    const Params P = tomo()->params;
    if (g == nullptr) return false;
    for (size_t i = 0; i < P.plans.size(); i++)
        if (g[i] == nullptr) {
            printf("planogram::apply_solid_angle_correction: Error data not set!\n");
            return false;
        }
    return stream_planograms(P, g, nullptr, "set_solid_angle_correction",
                             [&](const petl_geom& G, float* dg, float*, int b, int e, cudaStream_t st) {
                                 return petl::solid_angle(G, dg, do_inverse, b, e, st);
                             });
}

// PETL::apply_corrections (src/petl.cpp:163-192): g = g / r, then the
// bad-pixel median in-fill below threshold * median(r) per projection
bool apply_corrections(float** g, float** r, float threshold)
{
    const Params P = tomo()->params;
    if (g == nullptr || r == nullptr || P.plans.empty()) return false;
    for (size_t i = 0; i < P.plans.size(); i++)
        if (g[i] == nullptr || r[i] == nullptr) return false;
    return stream_planograms(P, g, r, "apply_corrections",
                             [&](const petl_geom& G, float* dg, float* dr, int b, int e, cudaStream_t st) {
                                 return petl::apply_corrections(G, dg, dr, threshold, b, e, st);
                             });
}

// ---------------------------------------------------------------------------
// projectors
// ---------------------------------------------------------------------------
bool project(float** g, float* f)
{
    const Params P = tomo()->params;
    if (g == nullptr || f == nullptr || !P.allDefined()) return false;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("project", cudaErrorNoDevice);
    DevBuf df;
    if (!df.alloc(P.volElems() * 4, c->compute)) return cuda_ok("project alloc", df.err);
    if (!cuda_ok("project H2D", copy_h2d(df.f(), f, P.volElems() * 4, c->compute)))
        return false;
    bool ok = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom G = P.full(i);
        const size_t slab = size_t(G.N_v0) * G.N_u1 * G.N_u0;
        DevBuf dg;
        if (!dg.alloc(slab * G.N_v1 * 4, c->compute)) return cuda_ok("project alloc", dg.err);
        // split kernels: each chunk of views goes back while the next computes
        ViewCopy vc{G, g[i], dg.f(), c->compute, c->copy, true};
        vc.pinned = host_pinned(g[i]);
        const petl::shear::ChunkHook hook{&ViewCopy::run, &vc};
        const int rc = petl::shear::project_chunked(G, df.f(), dg.f(), kChunkViews, hook, c->compute);
        vc.flush();
        const bool split = rc != petl::shear::kNotApplicable;
        if (split) ok = report("project", rc) && vc.ok;
        const int step = slab_step(G);
        for (int b = split ? G.N_v1 : 0; b < G.N_v1 && ok; b += step) {
            const int e = std::min(G.N_v1, b + step);
            ok = report("project", petl_project_range_dev(&G, df.f(), dg.f(), b, e, 0, 1, c->compute));
            cudaEvent_t ev;
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            cudaEventRecord(ev, c->compute);
            cudaStreamWaitEvent(c->copy, ev, 0);
            cudaEventDestroy(ev);
            ok = ok && cuda_ok("project D2H", copy_d2h(g[i] + size_t(b) * slab, dg.f() + size_t(b) * slab,
                                                       size_t(e - b) * slab * 4, c->copy));
        }
        // the buffer is released on the compute stream: order it after the copies
        cudaEvent_t done;
        cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
        cudaEventRecord(done, c->copy);
        cudaStreamWaitEvent(c->compute, done, 0);
        cudaEventDestroy(done);
    }
    ok = cuda_ok("project sync", cudaStreamSynchronize(c->copy)) && ok;
    ok = cuda_ok("project sync", cudaStreamSynchronize(c->compute)) && ok;
    return device_ok("project") && ok;
}

static bool backproject_impl(const Params& P, float** g, float* f, bool fbp_weight_unused)
{
    (void)fbp_weight_unused;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("backproject", cudaErrorNoDevice);
    DevBuf df;
    if (!df.alloc(P.volElems() * 4, c->compute)) return cuda_ok("backproject alloc", df.err);
    bool ok = true;
    bool first = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom G = P.full(i);
        const size_t slab = size_t(G.N_v0) * G.N_u1 * G.N_u0;
        DevBuf dg;
        if (!dg.alloc(slab * G.N_v1 * 4, c->compute)) return cuda_ok("backproject alloc", dg.err);
        // the copy stream may only start once the buffer exists on the compute stream
        cudaEvent_t ready;
        cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
        cudaEventRecord(ready, c->compute);
        cudaStreamWaitEvent(c->copy, ready, 0);
        cudaEventDestroy(ready);
        // split kernels: each chunk of views computes while the next comes in
        ViewCopy vc{G, g[i], dg.f(), c->compute, c->copy, false};
        const petl::shear::ChunkHook hook{&ViewCopy::run, &vc};
        const int rc = petl::shear::backproject_chunked(G, dg.f(), df.f(), PETL_BP_REFERENCE, first ? 0 : 1, 1.0f,
                                                        kChunkViews, hook, c->compute);
        const bool split = rc != petl::shear::kNotApplicable;
        if (split) {
            ok = report("backproject", rc) && vc.ok;
            first = false;
        }
        const int step = slab_step(G);
        for (int b = split ? G.N_v1 : 0; b < G.N_v1 && ok; b += step) {
            const int e = std::min(G.N_v1, b + step);
            ok = cuda_ok("backproject H2D", copy_h2d(dg.f() + size_t(b) * slab, g[i] + size_t(b) * slab,
                                                     size_t(e - b) * slab * 4,
                                                            c->copy));
            cudaEvent_t ev;
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            cudaEventRecord(ev, c->copy);
            cudaStreamWaitEvent(c->compute, ev, 0);
            cudaEventDestroy(ev);
            ok = ok && report("backproject", petl_backproject_range_dev(&G, dg.f(), df.f(), PETL_BP_REFERENCE,
                                                                        first ? 0 : 1, 1.0f, b, e, 0, 1, c->compute));
            first = false;
        }
    }
    ok = ok && cuda_ok("backproject D2H",
                       copy_d2h(f, df.f(), P.volElems() * 4, c->compute));
    ok = cuda_ok("backproject sync", cudaStreamSynchronize(c->compute)) && ok;
    return device_ok("backproject") && ok;
}

bool backproject(float** g, float* f)
{
    const Params P = tomo()->params;
    if (g == nullptr || f == nullptr || !P.allDefined()) return false;
    return backproject_impl(P, g, f, false);
}

bool FBP(float** g, float* f)
{
    const Params P = tomo()->params;
    if (g == nullptr || f == nullptr || !P.allDefined()) return false;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("FBP", cudaErrorNoDevice);
    DevBuf df;
    if (!df.alloc(P.volElems() * 4, c->compute)) return cuda_ok("FBP alloc", df.err);
    bool ok = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        const petl_geom G = P.full(i);
        const size_t n = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0;
        DevBuf dg;
        if (!dg.alloc(n * 4, c->compute)) return cuda_ok("FBP alloc", dg.err);
        ok = cuda_ok("FBP H2D", copy_h2d(dg.f(), g[i], n * 4, c->compute));
        // already-rebinned data is filtered and weighted in the caller's array,
        // as the reference does (src/petl.cpp:335-349)
        float* host_back = G.N_v1 == 1 ? g[i] : nullptr;
        ok = ok && report("FBP", petl::fbp(G, dg.f(), df.f(), i > 0 ? 1 : 0, c->compute, host_back));
    }
    ok = ok && cuda_ok("FBP D2H", copy_d2h(f, df.f(), P.volElems() * 4, c->compute));
    ok = cuda_ok("FBP sync", cudaStreamSynchronize(c->compute)) && ok;
    return device_ok("FBP") && ok;
}

bool PFDR(float** g, float** g_reb)
{
    Model* m = tomo();
    const Params P = m->params;
    if (g == nullptr || g_reb == nullptr || !P.geometryDefined()) return false;
    DevCtx* c = dev_ctx();
    if (!c) return cuda_ok("PFDR", cudaErrorNoDevice);
    bool ok = true;
    for (size_t i = 0; i < P.plans.size() && ok; i++) {
        petl_geom G = P.plans[i];
        // PFDR needs no volume; give the geometry check a nominal one
        petl_geom_set_volume(&G, 1, 1, 1, 1.0f, 1.0f, 0.f, 0.f, 0.f);
        const size_t n = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0;
        const size_t nr = size_t(G.N_v0) * G.N_u1 * G.N_u0;
        DevBuf dg, dr;
        if (!dg.alloc(n * 4, c->compute) || !dr.alloc(nr * 4, c->compute))
            return cuda_ok("PFDR alloc", dg.err != cudaSuccess ? dg.err : dr.err);
        ok = cuda_ok("PFDR H2D", copy_h2d(dg.f(), g[i], n * 4, c->compute));
        ok = ok && report("PFDR", petl_pfdr_dev(&G, dg.f(), dr.f(), c->compute));
        ok = ok && cuda_ok("PFDR D2H", copy_d2h(g_reb[i], dr.f(), nr * 4, c->compute));
        // PETL::doPFDR rewrites the model's planogram (src/petl.cpp:379-380)
        m->params.plans[i].N_v1 = 1;
        m->params.plans[i].v1_0 = 0.0f;
    }
    ok = cuda_ok("PFDR sync", cudaStreamSynchronize(c->compute)) && ok;
    return ok;
}

// ---------------------------------------------------------------------------
// elementwise on host arrays (src/petl_c_interface.cpp:313-469)
// ---------------------------------------------------------------------------
bool multiply3D(float* x, float* y, int N_1, int N_2, int N_3)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) { printf("multiply invalid inputs\n"); return false; }
    return binop(x, y, size_t(N_1) * N_2 * N_3, MULT);
}
bool multiply4D(float* x, float* y, int N_1, int N_2, int N_3, int N_4)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0 || N_4 <= 0) { printf("multiply invalid inputs\n"); return false; }
    return binop(x, y, size_t(N_1) * N_2 * N_3 * N_4, MULT);
}
bool divide3D(float* x, float* y, int N_1, int N_2, int N_3)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) { printf("divide invalid inputs\n"); return false; }
    return binop(x, y, size_t(N_1) * N_2 * N_3, DIV);
}
bool divide4D(float* x, float* y, int N_1, int N_2, int N_3, int N_4)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0 || N_4 <= 0) { printf("divide invalid inputs\n"); return false; }
    return binop(x, y, size_t(N_1) * N_2 * N_3 * N_4, DIV);
}
bool rdivide3D(float* num, float* denom, int N_1, int N_2, int N_3)
{
    if (!num || !denom || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) { printf("rdivide invalid inputs\n"); return false; }
    return binop(denom, num, size_t(N_1) * N_2 * N_3, RDIV);
}
bool rdivide4D(float* num, float* denom, int N_1, int N_2, int N_3, int N_4)
{
    if (!num || !denom || N_1 <= 0 || N_2 <= 0 || N_3 <= 0 || N_4 <= 0) { printf("rdivide invalid inputs\n"); return false; }
    return binop(denom, num, size_t(N_1) * N_2 * N_3 * N_4, RDIV);
}
static bool recip(float* x, size_t n, float v)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) x[i] = (x[i] == 0.0f) ? v : float(1.0 / x[i]);
    return true;
}
bool reciprocal3D(float* x, int N_1, int N_2, int N_3, float v)
{
    if (!x || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) { printf("rdivide invalid inputs\n"); return false; }
    return recip(x, size_t(N_1) * N_2 * N_3, v);
}
bool reciprocal4D(float* x, int N_1, int N_2, int N_3, int N_4, float v)
{
    if (!x || N_1 <= 0 || N_2 <= 0 || N_3 <= 0 || N_4 <= 0) { printf("rdivide invalid inputs\n"); return false; }
    return recip(x, size_t(N_1) * N_2 * N_3 * N_4, v);
}
float inner_product3D(float* x, float* y, float* w, int N_1, int N_2, int N_3)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) { printf("inner_product invalid inputs\n"); return 0.0f; }
    return inner(x, y, w, size_t(N_2) * N_3, size_t(N_1));
}
float inner_product4D(float* x, float* y, float* w, int N_1, int N_2, int N_3, int N_4)
{
    if (!x || !y || N_1 <= 0 || N_2 <= 0 || N_3 <= 0 || N_4 <= 0) { printf("inner_product invalid inputs\n"); return 0.0f; }
    // 4D: per 3D block a float result summed in double (src/data_cube.cpp:340-357)
    double acc = 0.0;
    const size_t blk = size_t(N_2) * N_3 * N_4;
    for (int i = 0; i < N_1; i++)
        acc += double(inner(x + i * blk, y + i * blk, w ? w + i * blk : nullptr, size_t(N_3) * N_4, size_t(N_2)));
    return float(acc);
}

// ---------------------------------------------------------------------------
// regularizers (src/petl_c_interface.cpp:487-531)
// ---------------------------------------------------------------------------
namespace {
struct Staged {
    // device copies of host arrays (or the caller's device pointers)
    float* d = nullptr;
    DevBuf buf;
    bool stage(float* p, size_t n, bool on_cpu, cudaStream_t st, bool copy_in = true)
    {
        if (!on_cpu) {
            d = p;
            return true;
        }
        if (!buf.alloc(n * 4, st)) return false;
        d = buf.f();
        return !copy_in || copy_h2d(d, p, n * 4, st) == cudaSuccess;
    }
};
double read_scalar(double* dptr, cudaStream_t st)
{
    double h = 0.0;
    cudaMemcpyAsync(&h, dptr, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return h;
}
}  // namespace

float TV_cost(float* f, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu)
{
    if (!f) return -1.0f;
    DevCtx* c = dev_ctx();
    if (!c) return -1.0f;
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf;
    DevBuf out;
    if (!sf.stage(f, n, data_on_cpu, c->compute) || !out.alloc(8, c->compute)) return -1.0f;
    if (!report("TV_cost", petl_tv_cost_dev(sf.d, N_1, N_2, N_3, delta, beta, p, 26, (double*)out.p, c->compute)))
        return -1.0f;
    return float(read_scalar((double*)out.p, c->compute));
}

bool TV_gradient(float* f, float* Df, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu)
{
    if (!f || !Df) return false;
    DevCtx* c = dev_ctx();
    if (!c) return false;
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf, sd;
    if (!sf.stage(f, n, data_on_cpu, c->compute) || !sd.stage(Df, n, data_on_cpu, c->compute, false)) return false;
    bool ok = report("TV_gradient", petl_tv_gradient_dev(sf.d, sd.d, N_1, N_2, N_3, delta, beta, p, 26, c->compute));
    if (ok && data_on_cpu) ok = cuda_ok("TV_gradient D2H", copy_d2h(Df, sd.d, n * 4, c->compute));
    return cuda_ok("TV_gradient sync", cudaStreamSynchronize(c->compute)) && ok;
}

float TV_quadForm(float* f, float* d, int N_1, int N_2, int N_3, float delta, float beta, float p, bool data_on_cpu)
{
    if (!f || !d) return -1.0f;
    DevCtx* c = dev_ctx();
    if (!c) return -1.0f;
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf, sd;
    DevBuf out;
    if (!sf.stage(f, n, data_on_cpu, c->compute) || !sd.stage(d, n, data_on_cpu, c->compute) || !out.alloc(8, c->compute))
        return -1.0f;
    if (!report("TV_quadForm",
                petl_tv_quadform_dev(sf.d, sd.d, N_1, N_2, N_3, delta, beta, p, 26, (double*)out.p, c->compute)))
        return -1.0f;
    return float(read_scalar((double*)out.p, c->compute));
}

// gradient-descent TV smoothing / denoising (src/total_variation.cu:813-935)
static bool tv_iterate(float* f, int N_1, int N_2, int N_3, float delta, float beta, float p, int numIter,
                       bool data_on_cpu, bool denoise)
{
    if (!f) return false;
    DevCtx* c = dev_ctx();
    if (!c) return false;
    if (delta < 1.0e-8) delta = float(1.0e-8);
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf;
    DevBuf dd, f0, sc;
    if (!sf.stage(f, n, data_on_cpu, c->compute) || !dd.alloc(n * 4, c->compute) || !sc.alloc(16, c->compute))
        return false;
    if (denoise) {
        if (!f0.alloc(n * 4, c->compute)) return false;
        cudaMemcpyAsync(f0.p, sf.d, n * 4, cudaMemcpyDeviceToDevice, c->compute);
    }
    bool ok = true;
    for (int it = 0; it < numIter && ok; it++) {
        ok = report("tv", petl_tv_gradient_dev(sf.d, dd.f(), N_1, N_2, N_3, delta, beta, p, 26, c->compute));
        ok = ok && report("tv", petl_dot_dev(dd.f(), dd.f(), nullptr, (long long)n, (double*)sc.p, c->compute));
        ok = ok && report("tv", petl_tv_quadform_dev(sf.d, dd.f(), N_1, N_2, N_3, delta, beta, p, 26,
                                                     (double*)sc.p + 1, c->compute));
        if (!ok) break;
        double h[2];
        cudaMemcpyAsync(h, sc.p, 16, cudaMemcpyDeviceToHost, c->compute);
        cudaStreamSynchronize(c->compute);
        const float num = float(h[0]), den = float(h[1]);
        if (den <= 1.0e-16) break;
        const float step = num / den;
        // f <- f - step*d  (diffuse);  f <- (1-step) f - step (d - f0)  (denoise)
        if (denoise) {
            ok = report("tv", petl_axpby_dev(sf.d, dd.f(), 1.0f - step, -step, (long long)n, c->compute));
            ok = ok && report("tv", petl_axpby_dev(sf.d, f0.f(), 1.0f, step, (long long)n, c->compute));
        } else {
            ok = report("tv", petl_axpby_dev(sf.d, dd.f(), 1.0f, -step, (long long)n, c->compute));
        }
    }
    if (ok && data_on_cpu) ok = cuda_ok("tv D2H", copy_d2h(f, sf.d, n * 4, c->compute));
    return cuda_ok("tv sync", cudaStreamSynchronize(c->compute)) && ok;
}

bool diffuse(float* f, int N_1, int N_2, int N_3, float delta, float p, int numIter, bool data_on_cpu)
{
    return tv_iterate(f, N_1, N_2, N_3, delta, 1.0f, p, numIter, data_on_cpu, false);
}

bool TV_denoise(float* f, int N_1, int N_2, int N_3, float delta, float beta, float p, int numIter, bool doMean,
                bool data_on_cpu)
{
    (void)doMean;  // the reference C ABI does not forward it (src/petl_c_interface.cpp:511-515)
    return tv_iterate(f, N_1, N_2, N_3, delta, beta, p, numIter, data_on_cpu, true);
}

bool relativeDifferences_gradient(float* f, float* Df, int N_1, int N_2, int N_3, float delta, float beta)
{
    if (f == nullptr || Df == nullptr || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) return false;
    DevCtx* c = dev_ctx();
    if (!c) return false;
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf, sd;
    if (!sf.stage(f, n, true, c->compute) || !sd.stage(Df, n, true, c->compute, false)) return false;
    bool ok = report("relativeDifferences_gradient",
                     petl_rd_gradient_dev(sf.d, sd.d, N_1, N_2, N_3, delta, beta, c->compute));
    ok = ok && cuda_ok("rd D2H", copy_d2h(Df, sd.d, n * 4, c->compute));
    return cuda_ok("rd sync", cudaStreamSynchronize(c->compute)) && ok;
}

bool gaussian_filter(float* f, int N_1, int N_2, int N_3, float FWHM, int numDims)
{
    if (f == nullptr || N_1 <= 0 || N_2 <= 0 || N_3 <= 0) return false;
    DevCtx* c = dev_ctx();
    if (!c) return false;
    const size_t n = size_t(N_1) * N_2 * N_3;
    Staged sf;
    if (!sf.stage(f, n, true, c->compute)) return false;
    bool ok = report("gaussian_filter", petl_gaussian_filter_dev(sf.d, N_1, N_2, N_3, FWHM, numDims, c->compute));
    ok = ok && cuda_ok("gauss D2H", copy_d2h(f, sf.d, n * 4, c->compute));
    return cuda_ok("gauss sync", cudaStreamSynchronize(c->compute)) && ok;
}

}  // extern "C"
