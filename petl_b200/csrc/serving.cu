// Reconstruction server: continuous batching of OSEM requests on one GPU.
//
// The reference serves reconstructions one call at a time through
// petl_server.py (src/petl_server.py:1534-1606), moving the planogram over
// PCIe on every iteration.  Here a worker thread owns the device:
//
//  * admission: a submitted request waits until its device footprint (data,
//    ratio, image, backprojection, projector scratch) fits the HBM budget next
//    to the requests already running and a slot is free; then its data is
//    copied in once and stays resident;
//  * requests of like geometry share their geometry's state: the per-subset
//    sensitivity images P_s^T 1 and the projector shift tables are computed
//    once per (geometry, subset count), kept in a cache that counts against
//    the budget (idle entries are evicted oldest first when memory is
//    needed), and reused by every later request of that geometry;
//  * continuous batching: every active request has its own CUDA stream, and
//    the worker keeps up to `depth` OSEM subset steps in flight per request,
//    issued oldest request first while the work in flight is under a cap of
//    about two full-size steps: large requests run nearly in arrival order
//    (the GPU is full with one of them), small ones overlap with them and
//    with each other, and new requests join while others run;
//  * batched launches: when a request of a geometry whose subset steps are
//    too small to fill the device issues a step with none in flight, up to
//    seven younger active requests of its geometry and subset count with no
//    step in flight join it, each at its own subset: one launch of each
//    projector kernel (and of the image update) serves them all, on the
//    first one's stream, ordered after and before each member's own stream
//    by events;
//  * completion: after the last step the image is copied to a pinned host
//    buffer, the device memory is returned to the stream-ordered pool and
//    the request's latency (submit to result on the host) is recorded;
//  * deadlines and cancellation: a request may carry a deadline (seconds
//    after submission) and may be cancelled; a pending one is dropped before
//    admission, an active one issues no further steps, its steps in flight
//    finish, its memory is released and its waiter gets an error.
//
// Each request runs the same kernels in the same order whatever else is
// running, so its result is bit-identical alone and in a mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "projector.cuh"
#include "shear.cuh"

namespace petl {
bool shear_eligible(const petl_geom& G);
int project_range(const petl_geom& G, const float* f, float* g, const ViewRange& vr, const float* meas,
                  cudaStream_t st);
int backproject_range(const petl_geom& G, const float* g, float* f, int mode, int accumulate, float scale,
                      const ViewRange& vr, cudaStream_t st);

namespace {

using Clock = std::chrono::steady_clock;

__global__ void k_fill(float* __restrict__ x, long long n, float v)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = v;
}

// zeros -> 1 (sensitivity normalisation of the reference MLEM)
__global__ void k_zero_to_one(float* __restrict__ x, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (x[i] == 0.0f) x[i] = 1.0f;
}

__device__ __forceinline__ void mlem_update(float* __restrict__ f, const float* __restrict__ d,
                                            const float* __restrict__ s, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float den = s[i];
        f[i] *= den == 0.0f ? 0.0f : d[i] / den;
    }
}

__global__ void k_mlem(float* __restrict__ f, const float* __restrict__ d, const float* __restrict__ s, long long n)
{
    mlem_update(f, d, s, n);
}

// the image updates of a batched step: member blockIdx.y
struct MlemMembers {
    float* f[shear::kMaxMembers];
    const float* d[shear::kMaxMembers];
    const float* s[shear::kMaxMembers];
};

__global__ void k_mlem_members(const MlemMembers P, long long n)
{
    const int b = blockIdx.y;
    mlem_update(shear::member_pick(P.f, b), shear::member_pick(P.d, b), shear::member_pick(P.s, b), n);
}

unsigned blocks_for(long long n) { return unsigned(std::min<long long>((n + 255) / 256, 148LL * 8)); }

enum State { kPending = 0, kActive = 1, kDone = 2, kFailed = 3 };

// Geometry state shared by the requests of one (geometry, subset count).
struct GeomState {
    std::string key;
    float* sens = nullptr;  // [subsets][numZ][numY][numX], zeros -> 1
    shear::TableBuf tables;
    bool shear = false;
    bool batch = false;  // split projector and small steps: requests share launches
    cudaEvent_t ready = nullptr;  // recorded after the state was computed
    size_t bytes = 0;
    int users = 0;
    unsigned long long last_use = 0;
};

std::string geom_key(const petl_geom& G, int subsets)
{
    std::string k(reinterpret_cast<const char*>(&G), sizeof(petl_geom));
    k.append(reinterpret_cast<const char*>(&subsets), sizeof(int));
    return k;
}

size_t state_bytes(const petl_geom& G, int subsets)
{
    const size_t nv = size_t(G.numX) * G.numY * G.numZ;
    return 4 * nv * size_t(subsets) + shear::table_bytes(G) + 4096;
}

// work of one subset step: rays x planes
double step_work(const petl_geom& G, int subsets)
{
    return double(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0 * double(G.numY) / double(subsets);
}

// A subset step whose forward z-tap launch has fewer CTAs than two waves of
// the SMs leaves most of the device idle: requests of its geometry share
// launches.  Larger steps fill the device alone, and batching them would
// only tie the requests' progress together.
bool small_step(const petl_geom& G, int subsets, int sms)
{
    const long long views = (G.N_v0 + subsets - 1) / subsets;
    const long long ctas = ((G.N_u0 + 63) / 64) * ((G.N_u1 + 31) / 32) * ((G.N_v1 + 15) / 16) * views;
    return ctas < 2LL * sms;
}

struct Request {
    long long id = 0;
    petl_geom G{};
    const float* g_host = nullptr;
    int subsets = 1, iters = 1;
    State state = kPending;
    std::string error;
    Clock::time_point t_submit, t_admit, t_done;
    bool has_deadline = false;
    Clock::time_point deadline;
    bool cancelled = false;  // set by petl_server_cancel under the server mutex
    size_t bytes = 0;
    // device state
    cudaStream_t st = nullptr;
    float *g = nullptr, *ratio = nullptr, *f = nullptr, *d = nullptr;
    std::shared_ptr<GeomState> gs;  // sensitivities and tables of the geometry
    double work = 0;                // of one subset step
    int steps_total = 0, steps_issued = 0;
    std::deque<cudaEvent_t> inflight;  // one event per issued step
    cudaEvent_t result_ev = nullptr;
    float* out_host = nullptr;  // pinned
    bool result_issued = false;
};

size_t footprint(const petl_geom& G, int subsets)
{
    const size_t ng = size_t(G.N_v1) * G.N_v0 * G.N_u1 * G.N_u0, nv = size_t(G.numX) * G.numY * G.numZ;
    // the split projector's scratch for the views of one subset step (one
    // volume-sized FP32 array per view, capped by the per-call budget)
    const size_t views = (size_t(G.N_v0) + size_t(subsets) - 1) / size_t(subsets);
    const size_t per_view = size_t(G.numY) * G.numZ * ((size_t(G.N_u0) + 3) & ~size_t(3)) * 4;
    const size_t scratch = std::min(views * per_view, std::max(per_view, shear::split_scratch_budget()));
    return 4 * (2 * ng + 2 * nv) + scratch + (size_t(1) << 20);
}

}  // namespace

struct Server {
    int device = 0;
    double budget = 0;
    int max_active = 1, depth = 2;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    long long next_id = 1;
    std::deque<std::shared_ptr<Request>> pending;
    std::vector<std::shared_ptr<Request>> active;
    std::map<long long, std::shared_ptr<Request>> all;
    double in_use = 0, peak = 0;
    long long completed = 0, failed = 0;
    std::thread worker;
    // geometry states (worker thread only; their bytes count in in_use)
    std::map<std::string, std::shared_ptr<GeomState>> states;
    unsigned long long use_clock = 0;
    cudaStream_t aux = nullptr;  // frees evicted states
    double work_cap = 0;
    // reused per-request resources: streams (worker thread only) and pinned
    // result buffers by size (worker and waiters, under pool_mu); creating
    // a stream and page-locking a result per request cost milliseconds of
    // the worker's time each
    std::vector<cudaStream_t> free_streams;
    std::mutex pool_mu;
    std::multimap<size_t, float*> free_host;
    size_t free_host_bytes = 0;

    float* take_host(size_t bytes)
    {
        {
            std::lock_guard<std::mutex> lk(pool_mu);
            auto it = free_host.find(bytes);
            if (it != free_host.end()) {
                float* p = it->second;
                free_host.erase(it);
                free_host_bytes -= bytes;
                return p;
            }
        }
        float* p = nullptr;
        return cudaHostAlloc(reinterpret_cast<void**>(&p), bytes, cudaHostAllocDefault) == cudaSuccess ? p : nullptr;
    }
    void give_host(float* p, size_t bytes)
    {
        if (!p) return;
        std::lock_guard<std::mutex> lk(pool_mu);
        if (free_host_bytes + bytes > (size_t(4) << 30)) {  // keep at most 4 GB page-locked
            cudaFreeHost(p);
            return;
        }
        free_host.emplace(bytes, p);
        free_host_bytes += bytes;
    }

    void run();
    void drop_expired_pending();
    bool evict_idle_states(double need);
    bool build_state(Request& r, GeomState& e);
    bool admit(Request& r);
    bool issue_step(Request& r);
    bool issue_batch(std::vector<Request*>& ms);
    void release(Request& r);
    // batched launches: members per step at most (1: none), and counts
    // batched steps off by default: on the serving workload they measured
    // the same throughput as separate streams and a higher p99
    std::atomic<int> batch_max{1};
    int sms = 148;  // multiprocessors of the device
    std::atomic<long long> batched_steps{0}, batched_members{0};
    void fail(Request& r, const std::string& why);
};

namespace {

int stream_for(cudaStream_t* st)
{
    return cudaStreamCreateWithFlags(st, cudaStreamNonBlocking) == cudaSuccess ? 0 : -1;
}

}  // namespace

void Server::fail(Request& r, const std::string& why)
{
    r.error = why;
    r.state = kFailed;
}

// A request's reason to stop, or nullptr: cancelled, or past its deadline.
const char* stop_reason(const Request& r, Clock::time_point now)
{
    if (r.cancelled) return "cancelled";
    if (r.has_deadline && now >= r.deadline) return "deadline exceeded";
    return nullptr;
}

// Pending requests that were cancelled or whose deadline passed fail
// without being admitted (caller holds the mutex).
void Server::drop_expired_pending()
{
    const Clock::time_point now = Clock::now();
    for (auto it = pending.begin(); it != pending.end();) {
        Request& r = **it;
        if (const char* why = stop_reason(r, now)) {
            fail(r, std::string(why) + " before admission");
            r.t_done = now;
            failed++;
            it = pending.erase(it);
            cv_done.notify_all();
        } else {
            ++it;
        }
    }
}

// Frees idle geometry states, least recently used first, until `need` more
// bytes fit the budget; false if they cannot be made to fit.
bool Server::evict_idle_states(double need)
{
    while (in_use + need > budget) {
        std::shared_ptr<GeomState> victim;
        for (auto& kv : states)
            if (kv.second->users == 0 && (!victim || kv.second->last_use < victim->last_use)) victim = kv.second;
        if (!victim) return false;
        // its users have finished (their streams were synchronised): free it
        if (victim->sens) cudaFreeAsync(victim->sens, aux);
        if (victim->tables.base) cudaFreeAsync(victim->tables.base, aux);
        if (victim->ready) cudaEventDestroy(victim->ready);
        in_use -= double(victim->bytes);
        states.erase(victim->key);
    }
    return true;
}

// Sensitivities P_s^T 1 (zeros -> 1) and tables of a geometry, on the
// stream of the request that first needs them.
bool Server::build_state(Request& r, GeomState& e)
{
    const petl_geom& G = r.G;
    const long long ng = (long long)G.N_v1 * G.N_v0 * G.N_u1 * G.N_u0;
    const long long nv = (long long)G.numX * G.numY * G.numZ;
    bool ok = scratch_alloc(reinterpret_cast<void**>(&e.sens), nv * 4 * r.subsets, r.st) == cudaSuccess;
    e.shear = shear_eligible(G);
    e.batch = e.shear && small_step(G, r.subsets, sms);
    if (ok && e.shear) ok = shear::make_tables(G, e.tables, r.st) == 0;
    if (!ok) return false;
    k_fill<<<blocks_for(ng), 256, 0, r.st>>>(r.ratio, ng, 1.0f);
    note_launch();
    for (int s = 0; s < r.subsets && ok; s++) {
        const ViewRange vr{0, G.N_v1, s, r.subsets};
        float* sv = e.sens + size_t(s) * nv;
        const int rc = e.shear ? shear::backproject_with(G, r.ratio, sv, PETL_BP_REFERENCE, 0, 1.0f, vr, e.tables.T, r.st)
                               : backproject_range(G, r.ratio, sv, PETL_BP_REFERENCE, 0, 1.0f, vr, r.st);
        ok = rc == 0;
        k_zero_to_one<<<blocks_for(nv), 256, 0, r.st>>>(sv, nv);
        note_launch();
    }
    return ok && cudaEventCreateWithFlags(&e.ready, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventRecord(e.ready, r.st) == cudaSuccess;
}

bool Server::admit(Request& r)
{
    // device buffers and the data copy, all on the request's stream
    const petl_geom& G = r.G;
    const long long ng = (long long)G.N_v1 * G.N_v0 * G.N_u1 * G.N_u0;
    const long long nv = (long long)G.numX * G.numY * G.numZ;
    if (!free_streams.empty()) {
        r.st = free_streams.back();
        free_streams.pop_back();
    } else if (stream_for(&r.st)) {
        fail(r, "cannot create a stream");
        return false;
    }
    r.out_host = take_host(size_t(nv) * 4);
    bool ok = scratch_alloc(reinterpret_cast<void**>(&r.g), ng * 4, r.st) == cudaSuccess &&
              scratch_alloc(reinterpret_cast<void**>(&r.ratio), ng * 4, r.st) == cudaSuccess &&
              scratch_alloc(reinterpret_cast<void**>(&r.f), nv * 4, r.st) == cudaSuccess &&
              scratch_alloc(reinterpret_cast<void**>(&r.d), nv * 4, r.st) == cudaSuccess && r.out_host != nullptr;
    if (!ok) {
        cudaGetLastError();
        fail(r, "admission failed: out of memory");
        return false;
    }
    // the geometry's shared state: reuse it, or build it here
    const std::string key = geom_key(G, r.subsets);
    auto it = states.find(key);
    if (it != states.end()) {
        r.gs = it->second;
        r.gs->users++;  // released in release()
        ok = cudaStreamWaitEvent(r.st, r.gs->ready, 0) == cudaSuccess;
    } else {
        auto e = std::make_shared<GeomState>();
        e->key = key;
        e->bytes = state_bytes(G, r.subsets);
        {
            std::lock_guard<std::mutex> lk(mu);
            in_use += double(e->bytes);
        }
        ok = build_state(r, *e);
        if (ok) {
            states[key] = e;
            r.gs = e;
            r.gs->users++;  // released in release()
        } else {
            if (e->sens) cudaFreeAsync(e->sens, r.st);
            if (e->tables.base) cudaFreeAsync(e->tables.base, r.st);
            if (e->ready) cudaEventDestroy(e->ready);
            std::lock_guard<std::mutex> lk(mu);
            in_use -= double(e->bytes);
        }
    }
    ok = ok && cudaMemcpyAsync(r.g, r.g_host, ng * 4, cudaMemcpyHostToDevice, r.st) == cudaSuccess;
    if (!ok) {
        fail(r, "admission failed: " + std::string(cudaGetErrorString(cudaGetLastError())));
        return false;
    }
    r.gs->last_use = ++use_clock;
    // image starts at 1
    k_fill<<<blocks_for(nv), 256, 0, r.st>>>(r.f, nv, 1.0f);
    note_launch();
    r.work = step_work(G, r.subsets);
    r.steps_total = r.iters * r.subsets;
    r.state = kActive;
    r.t_admit = Clock::now();
    return true;
}

bool Server::issue_step(Request& r)
{
    const petl_geom& G = r.G;
    const long long nv = (long long)G.numX * G.numY * G.numZ;
    const int s = r.steps_issued % r.subsets;
    const ViewRange vr{0, G.N_v1, s, r.subsets};
    const GeomState& e = *r.gs;
    int rc = e.shear ? shear::project_with(G, r.f, r.ratio, vr, r.g, e.tables.T, r.st)
                     : project_range(G, r.f, r.ratio, vr, r.g, r.st);
    if (!rc)
        rc = e.shear ? shear::backproject_with(G, r.ratio, r.d, PETL_BP_REFERENCE, 0, 1.0f, vr, e.tables.T, r.st)
                     : backproject_range(G, r.ratio, r.d, PETL_BP_REFERENCE, 0, 1.0f, vr, r.st);
    if (rc) {
        fail(r, "OSEM step failed");
        return false;
    }
    k_mlem<<<blocks_for(nv), 256, 0, r.st>>>(r.f, r.d, e.sens + size_t(s) * nv, nv);
    note_launch();
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, r.st);
    r.inflight.push_back(ev);
    r.steps_issued++;
    return true;
}

// One OSEM subset step for each of ms (same geometry state, split
// projector): the members' steps share one launch of each kernel on the
// first member's stream.  Each member's own stream is ordered before the
// batch (an event per member) and after it (its step event).  Where the
// batched kernels do not apply (scratch for all members' views), the
// members' steps are issued one by one on the same stream; every member's
// floats are those of its own step either way.
bool Server::issue_batch(std::vector<Request*>& ms)
{
    if (ms.size() == 1) return issue_step(*ms[0]);
    Request& L = *ms[0];
    const petl_geom& G = L.G;
    const GeomState& e = *L.gs;
    const int S = L.subsets;
    const long long nv = (long long)G.numX * G.numY * G.numZ;
    const int nb = int(ms.size());
    bool ok = true;
    for (int b = 1; b < nb && ok; b++) {
        cudaEvent_t ev;
        ok = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) break;
        ok = cudaEventRecord(ev, ms[b]->st) == cudaSuccess && cudaStreamWaitEvent(L.st, ev, 0) == cudaSuccess;
        cudaEventDestroy(ev);
    }
    shear::Members F, B;
    F.nb = B.nb = nb;
    MlemMembers U{};
    for (int b = 0; b < nb; b++) {
        Request& q = *ms[b];
        const int s = q.steps_issued % S;
        F.first[b] = B.first[b] = s;
        F.nv[b] = B.nv[b] = ViewRange{0, G.N_v1, s, S}.n_v0(G.N_v0);
        F.in[b] = q.f;
        F.out[b] = q.ratio;
        F.meas[b] = q.g;
        B.in[b] = q.ratio;
        B.out[b] = q.d;
        U.f[b] = q.f;
        U.d[b] = q.d;
        U.s[b] = e.sens + size_t(s) * nv;
    }
    const ViewRange vr{0, G.N_v1, 0, S};
    // the split kernels where a step of its own would take them (dispatch 2
    // and 3 force other kernel families)
    const bool split = dispatch_mode() != 2 && dispatch_mode() != 3;
    int rc = !ok ? -1 : split ? shear::project_split_members(G, F, vr, e.tables.T, L.st) : shear::kNotApplicable;
    if (rc == shear::kNotApplicable)
        for (int b = 0; b < nb && (rc == 0 || rc == shear::kNotApplicable); b++) {
            const ViewRange vb{0, G.N_v1, F.first[b], S};
            rc = shear::project_with(G, ms[b]->f, ms[b]->ratio, vb, ms[b]->g, e.tables.T, L.st);
        }
    if (rc == 0)
        rc = split ? shear::backproject_split_members(G, B, PETL_BP_REFERENCE, 0, 1.0f, vr, e.tables.T, L.st)
                   : shear::kNotApplicable;
    if (rc == shear::kNotApplicable)
        for (int b = 0; b < nb && (rc == 0 || rc == shear::kNotApplicable); b++) {
            const ViewRange vb{0, G.N_v1, B.first[b], S};
            rc = shear::backproject_with(G, ms[b]->ratio, ms[b]->d, PETL_BP_REFERENCE, 0, 1.0f, vb, e.tables.T,
                                         L.st);
        }
    if (rc) {
        for (Request* q : ms) fail(*q, "OSEM step failed");
        return false;
    }
    k_mlem_members<<<dim3(blocks_for(nv), unsigned(nb)), 256, 0, L.st>>>(U, nv);
    note_launch();
    cudaEvent_t done;
    cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    cudaEventRecord(done, L.st);
    L.inflight.push_back(done);
    for (int b = 1; b < nb; b++) {
        Request& q = *ms[b];
        cudaStreamWaitEvent(q.st, done, 0);
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        cudaEventRecord(ev, q.st);
        q.inflight.push_back(ev);
    }
    for (Request* q : ms) q->steps_issued++;
    batched_steps++;
    batched_members += nb;
    return true;
}

void Server::release(Request& r)
{
    for (cudaEvent_t e : r.inflight) cudaEventDestroy(e);
    r.inflight.clear();
    if (r.result_ev) cudaEventDestroy(r.result_ev);
    r.result_ev = nullptr;
    if (r.st) {
        if (r.g) cudaFreeAsync(r.g, r.st);
        if (r.ratio) cudaFreeAsync(r.ratio, r.st);
        if (r.f) cudaFreeAsync(r.f, r.st);
        if (r.d) cudaFreeAsync(r.d, r.st);
        cudaStreamSynchronize(r.st);
        free_streams.push_back(r.st);
    }
    if (r.gs) r.gs->users--;  // the use taken in admit()
    r.gs = nullptr;
    r.g = r.ratio = r.f = r.d = nullptr;
    r.st = nullptr;
}

void Server::run()
{
    cudaSetDevice(device);
    cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    while (true) {
        std::vector<std::shared_ptr<Request>> to_admit;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop) break;
            drop_expired_pending();
            // admission by HBM budget and free slots, in arrival order; a
            // geometry seen before needs no new state
            while (!pending.empty() && int(active.size() + to_admit.size()) < max_active) {
                auto& r = pending.front();
                bool known = states.count(geom_key(r->G, r->subsets)) != 0;
                for (auto& q : to_admit) known = known || (q->G.N_v0 == r->G.N_v0 &&
                                                            geom_key(q->G, q->subsets) == geom_key(r->G, r->subsets));
                const double need = double(r->bytes) + (known ? 0.0 : double(state_bytes(r->G, r->subsets)));
                const bool alone = active.empty() && to_admit.empty();
                if (in_use + need > budget && !evict_idle_states(need) && !alone) break;
                in_use += double(r->bytes);
                peak = std::max(peak, in_use + (known ? 0.0 : double(state_bytes(r->G, r->subsets))));
                to_admit.push_back(r);
                pending.pop_front();
            }
        }
        for (auto& r : to_admit) {
            if (!admit(*r)) {
                release(*r);
                std::lock_guard<std::mutex> lk(mu);
                in_use -= double(r->bytes);
                failed++;
                r->t_done = Clock::now();
                cv_done.notify_all();
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            active.push_back(r);
        }
        bool progressed = !to_admit.empty();
        // retire finished steps
        for (auto& rp : active) {
            Request& r = *rp;
            while (!r.inflight.empty() && cudaEventQuery(r.inflight.front()) == cudaSuccess) {
                cudaEventDestroy(r.inflight.front());
                r.inflight.pop_front();
                progressed = true;
            }
        }
        // issue new steps, oldest request first, while the work in flight is
        // under the cap (the oldest request may always keep `depth` steps)
        double inflight_work = 0;
        double biggest = 0;
        for (auto& rp : active) {
            inflight_work += double(rp->inflight.size()) * rp->work;
            biggest = std::max(biggest, rp->work);
        }
        const double cap = std::max(work_cap, 2.0 * biggest);
        const Clock::time_point now = Clock::now();
        bool oldest = true;
        auto can_step = [&](const Request& q) {
            return q.state == kActive && !q.result_issued && q.steps_issued < q.steps_total &&
                   int(q.inflight.size()) < depth;
        };
        for (size_t ai = 0; ai < active.size(); ai++) {
            Request& r = *active[ai];
            if (r.state == kActive && !r.result_issued) {
                const char* why = nullptr;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    why = stop_reason(r, now);
                }
                if (why) {  // no further steps; release() waits for those in flight
                    fail(r, why);
                    progressed = true;
                    continue;
                }
            }
            while (can_step(r) && (oldest || inflight_work + r.work <= cap)) {
                // younger requests of the same geometry state join this one's
                // launches (small steps of the split projector only) when
                // neither has a step in flight: the batch then waits on no
                // other stream, and no chain of batches ties the streams
                // together (a leader with steps in flight measured 0.6x the
                // throughput of unbatched steps at 200 small requests/s)
                std::vector<Request*> ms{&r};
                double w = r.work;
                if (batch_max > 1 && r.gs && r.gs->batch && r.inflight.empty())
                    for (size_t aj = ai + 1; aj < active.size() && int(ms.size()) < batch_max; aj++) {
                        Request& q = *active[aj];
                        if (q.gs != r.gs || !can_step(q) || !q.inflight.empty() || inflight_work + w + q.work > cap)
                            continue;
                        bool stopping = false;
                        {
                            std::lock_guard<std::mutex> lk(mu);
                            stopping = stop_reason(q, now) != nullptr;
                        }
                        if (stopping) continue;  // failed when the loop reaches it
                        ms.push_back(&q);
                        w += q.work;
                    }
                if (!issue_batch(ms)) break;
                inflight_work += w;
                progressed = true;
            }
            if (r.state == kActive) oldest = false;
            if (r.state == kActive && !r.result_issued && r.steps_issued == r.steps_total) {
                const long long nv = (long long)r.G.numX * r.G.numY * r.G.numZ;
                cudaMemcpyAsync(r.out_host, r.f, nv * 4, cudaMemcpyDeviceToHost, r.st);
                cudaEventCreateWithFlags(&r.result_ev, cudaEventDisableTiming);
                cudaEventRecord(r.result_ev, r.st);
                r.result_issued = true;
                progressed = true;
            }
        }
        // completions
        std::vector<std::shared_ptr<Request>> finished;
        for (auto& rp : active) {
            Request& r = *rp;
            const bool failed_now = r.state == kFailed;
            const bool done = r.result_issued && cudaEventQuery(r.result_ev) == cudaSuccess;
            if (done || failed_now) finished.push_back(rp);
        }
        for (auto& rp : finished) {
            Request& r = *rp;
            release(r);
            std::lock_guard<std::mutex> lk(mu);
            if (r.state != kFailed) {
                r.state = kDone;
                completed++;
            } else {
                failed++;
            }
            r.t_done = Clock::now();
            in_use -= double(r.bytes);
            active.erase(std::find(active.begin(), active.end(), rp));
            cv_done.notify_all();
            progressed = true;
        }
        if (!progressed) {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && pending.empty())
                cv_work.wait(lk, [&] { return stop || !pending.empty(); });
            else if (active.empty())
                // pending requests that do not fit yet cannot exist with no
                // request active; wake up for deadlines and cancellations
                cv_work.wait_for(lk, std::chrono::milliseconds(5));
            else if (!active.empty()) {
                // wait for the oldest step of some request instead of spinning
                lk.unlock();
                for (auto& rp : active)
                    if (!rp->inflight.empty()) {
                        cudaEventSynchronize(rp->inflight.front());
                        break;
                    }
            }
        }
    }
    // shutdown: drop whatever is left
    for (auto& rp : active) release(*rp);
    for (auto& rp : pending) rp->state = kFailed;
    for (auto& kv : states) {
        if (kv.second->sens) cudaFreeAsync(kv.second->sens, aux);
        if (kv.second->tables.base) cudaFreeAsync(kv.second->tables.base, aux);
        if (kv.second->ready) cudaEventDestroy(kv.second->ready);
    }
    states.clear();
    if (aux) {
        cudaStreamSynchronize(aux);
        cudaStreamDestroy(aux);
    }
    for (cudaStream_t st : free_streams) cudaStreamDestroy(st);
    free_streams.clear();
}

}  // namespace petl

using namespace petl;

extern "C" {

void* petl_server_create(double hbm_budget_bytes, int max_active, int depth, int device)
{
    clear_error();
    if (hbm_budget_bytes <= 0 || max_active < 1 || depth < 1) {
        set_error("server_create: invalid arguments");
        return nullptr;
    }
    Server* s = new Server();
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->depth = depth;
    s->worker = std::thread([s] { s->run(); });
    return s;
}

int petl_server_submit_deadline(void* server, const petl_geom* G, const float* g_host, int num_subsets, int num_iter,
                                double deadline_s, long long* id_out);

int petl_server_submit(void* server, const petl_geom* G, const float* g_host, int num_subsets, int num_iter,
                       long long* id_out)
{
    return petl_server_submit_deadline(server, G, g_host, num_subsets, num_iter, -1.0, id_out);
}

int petl_server_submit_deadline(void* server, const petl_geom* G, const float* g_host, int num_subsets, int num_iter,
                                double deadline_s, long long* id_out)
{
    clear_error();
    Server* s = static_cast<Server*>(server);
    std::string why;
    PETL_REQUIRE(s && G && g_host && id_out && num_subsets >= 1 && num_iter >= 1 && geom_valid(G, &why),
                 "server_submit: invalid arguments " + why);
    PETL_REQUIRE(num_subsets <= G->N_v0, "server_submit: more subsets than views");
    auto r = std::make_shared<Request>();
    r->G = *G;
    r->g_host = g_host;
    r->subsets = num_subsets;
    r->iters = num_iter;
    r->bytes = footprint(*G, num_subsets);
    r->t_submit = Clock::now();
    if (deadline_s >= 0.0) {
        r->has_deadline = true;
        r->deadline = r->t_submit + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(deadline_s));
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        PETL_REQUIRE(double(r->bytes + state_bytes(*G, num_subsets)) <= s->budget,
                     "server_submit: request larger than the HBM budget");
        r->id = s->next_id++;
        s->pending.push_back(r);
        s->all[r->id] = r;
        *id_out = r->id;
    }
    s->cv_work.notify_one();
    return 0;
}

int petl_server_wait(void* server, long long id, float* f_host, double* latency_s, double* queue_s)
{
    clear_error();
    Server* s = static_cast<Server*>(server);
    PETL_REQUIRE(s, "server_wait: null server");
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->all.find(id);
        PETL_REQUIRE(it != s->all.end(), "server_wait: unknown request");
        r = it->second;
        s->cv_done.wait(lk, [&] { return r->state == kDone || r->state == kFailed; });
        s->all.erase(it);
    }
    const double lat = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    const double q = r->state == kDone ? std::chrono::duration<double>(r->t_admit - r->t_submit).count() : lat;
    if (latency_s) *latency_s = lat;
    if (queue_s) *queue_s = q;
    int rc = 0;
    if (r->state == kDone) {
        if (f_host) std::memcpy(f_host, r->out_host, sizeof(float) * size_t(r->G.numX) * r->G.numY * r->G.numZ);
    } else {
        set_error("server request failed: " + r->error);
        rc = -1;
    }
    s->give_host(r->out_host, sizeof(float) * size_t(r->G.numX) * r->G.numY * r->G.numZ);
    r->out_host = nullptr;
    return rc;
}

int petl_server_cancel(void* server, long long id)
{
    clear_error();
    Server* s = static_cast<Server*>(server);
    PETL_REQUIRE(s, "server_cancel: null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->all.find(id);
        PETL_REQUIRE(it != s->all.end(), "server_cancel: unknown request");
        it->second->cancelled = true;
    }
    s->cv_work.notify_one();
    return 0;
}

// out[0..5] = completed, failed, active, pending, HBM bytes in use, peak HBM bytes reserved
int petl_server_set_batching(void* server, int max_members)
{
    Server* s = static_cast<Server*>(server);
    if (!s || max_members < 1 || max_members > shear::kMaxMembers) {
        set_error("server_set_batching: invalid arguments");
        return -1;
    }
    s->batch_max = max_members;
    return 0;
}

int petl_server_batch_stats(void* server, double* out)
{
    Server* s = static_cast<Server*>(server);
    if (!s || !out) return -1;
    out[0] = double(s->batched_steps.load());
    out[1] = double(s->batched_members.load());
    return 0;
}

int petl_server_stats(void* server, double* out)
{
    Server* s = static_cast<Server*>(server);
    if (!s || !out) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = double(s->completed);
    out[1] = double(s->failed);
    out[2] = double(s->active.size());
    out[3] = double(s->pending.size());
    out[4] = s->in_use;
    out[5] = s->peak;
    return 0;
}

void petl_server_destroy(void* server)
{
    Server* s = static_cast<Server*>(server);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->all)
        if (kv.second->out_host) cudaFreeHost(kv.second->out_host);
    for (auto& kv : s->free_host) cudaFreeHost(kv.second);
    delete s;
}

}  // extern "C"
