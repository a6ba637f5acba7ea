// Serving loop: continuous batching of fracture solves on one GPU.
//
// Requests (a scene description, its particles and a horizon in substeps)
// queue on submit.  Each gmpm_server_step admits queued requests in arrival
// order while the device-memory budget allows, advances every live scene
// together through one batch (one CUDA graph launch per substep), never past a
// scene's horizon, and retires scenes that reached it: their final fields
// are copied to host memory and their device memory is freed, so waiting
// requests can be admitted on the next step.  The batch is rebuilt whenever
// the live set changes; the launch shapes tuned for the first batch are
// reused.  Results do not depend on which scenes share a batch (bitwise in
// deterministic mode).  No reference counterpart: the reference runs one
// scene per process from its GLUT loop (gl_main.cpp:304-314).
//
// Threads: one thread steps the server; submit, poll, read, release and
// stats may be called from other threads at the same time (a mutex guards
// the queue, the request table and the counters; creating, advancing and
// retiring scenes run outside it).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "scene.h"

namespace gmpm {
namespace {

#define SERVE_TRY(expr)                                   \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return cuda_status(e_);    \
    } while (0)

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Fields kept for a finished request (original particle order, FP32).
constexpr int kKeptFields[] = {GMPM_FIELD_POSITION, GMPM_FIELD_VELOCITY, GMPM_FIELD_F, GMPM_FIELD_DAMAGE};

int kept_components(int field) {
    switch (field) {
        case GMPM_FIELD_POSITION:
        case GMPM_FIELD_VELOCITY: return 3;
        case GMPM_FIELD_F: return 9;
        case GMPM_FIELD_DAMAGE: return 1;
        default: return 0;
    }
}

struct Request {
    int64_t id = 0;
    gmpm_scene_desc desc{};
    std::vector<double> pos, vel, mass;
    std::vector<int32_t> mat;
    int64_t n = 0;
    int64_t horizon = 0;
    int64_t done = 0;
    int state = GMPM_REQUEST_QUEUED;
    gmpm_status status = GMPM_OK;
    size_t est_bytes = 0, bytes = 0;
    double t_submit = 0, t_admit = 0, t_finish = 0;
    gmpm_scene* scene = nullptr;
    // final fields (FP32, original order) in a pinned buffer: position,
    // velocity, F, damage at the offsets below, then the status flags
    unsigned char* results = nullptr;
    size_t results_bytes = 0;
    size_t offset[4] = {0, 0, 0, 0};
    unsigned int* flags = nullptr;
    cudaEvent_t ready = nullptr;  // the reads of a retiring request have landed
};

// Reused pinned host buffers: allocating pinned memory can stall the device,
// so buffers are kept and handed out again by size.
struct PinnedPool {
    std::multimap<size_t, unsigned char*> free_bufs;
    std::vector<unsigned char*> all;
    ~PinnedPool() {
        for (unsigned char* p : all) cudaFreeHost(p);
    }
    unsigned char* acquire(size_t bytes, size_t* got) {
        auto it = free_bufs.lower_bound(bytes);
        if (it != free_bufs.end() && it->first <= 2 * bytes + (1u << 20)) {
            unsigned char* p = it->second;
            *got = it->first;
            free_bufs.erase(it);
            return p;
        }
        size_t sz = 1u << 20;
        while (sz < bytes) sz <<= 1;
        unsigned char* p = nullptr;
        if (cudaMallocHost(reinterpret_cast<void**>(&p), sz) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        all.push_back(p);
        *got = sz;
        return p;
    }
    void release(unsigned char* p, size_t bytes) {
        if (p) free_bufs.emplace(bytes, p);
    }
};

// Device bytes of a scene before it exists: particle planes (55 words + 2 ids
// per particle in FP32, twice that in FP64), binning (3 words per particle and
// 10 bytes per page of the key space) and the page tiles/grid, with slack.
size_t estimate_bytes(const gmpm_scene_desc& d, int64_t n) {
    const size_t real = d.precision == GMPM_PRECISION_FP64 ? 8 : 4;
    const size_t per_particle = 55 * real + 8 + 12;
    size_t key_space = 1;
    for (int a = 0; a < 3; ++a) key_space *= (size_t)((d.grid_res[a] + 3) / 4 + 1);
    const size_t pages = (size_t)n / 64 + 256;
    return (size_t)n * per_particle + key_space * 10 + pages * 2 * (9 * 216 + 5 * 64 * 8) * real + (16u << 20);
}

}  // namespace

struct Server {
    gmpm_context* ctx = nullptr;
    gmpm_server_options opt{};
    std::mutex mu;  // reqs, queue, st and the request fields poll reads
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::deque<int64_t> queue;
    std::vector<Request*> live;  // stepping thread only
    std::vector<Request*> retiring;  // reads enqueued, waiting for their event (stepping thread only)
    std::vector<cudaEvent_t> spare_events;
    PinnedPool pinned;  // guarded by mu
    gmpm_batch* batch = nullptr;
    bool batch_stale = true;
    bool tuned = false;
    gmpm_batch_options tuned_opt{};
    int tuned_share[3] = {0, 0, 0};  // SMs per scene by size class, from the first tuned batch
    int64_t next_id = 1;
    size_t used = 0;
    gmpm_server_stats st{};
    double t0 = now_s();

    ~Server() {
        for (Request* r : retiring) cudaEventSynchronize(r->ready);
        for (cudaEvent_t e : spare_events) cudaEventDestroy(e);
        for (auto& kv : reqs)
            if (kv.second->ready) cudaEventDestroy(kv.second->ready);
        if (batch) gmpm_batch_destroy(batch);
        batch = nullptr;
        for (auto& kv : reqs)
            if (kv.second->scene) gmpm_scene_destroy(kv.second->scene);
    }

    void drop_batch() {
        if (batch) {
            gmpm_batch_info info;
            if (gmpm_batch_get_info(batch, &info) == GMPM_OK) {
                std::lock_guard<std::mutex> lk(mu);
                st.capture_microseconds += (int64_t)(info.capture_seconds * 1e6);
            }
            // only the first batch is tuned: if it ends before tuning finished,
            // later batches keep the default launch shapes
            remember_tuning();
            if (!tuned) {
                tuned = true;
                tuned_opt = gmpm_batch_options{};
            }
            batch_destroy_deferred(batch);
        }
        batch = nullptr;
        batch_stale = true;
    }

    gmpm_status submit(const gmpm_scene_desc* d, const gmpm_particle_init* init, int64_t horizon, int64_t* id) {
        if (!d || !init || !id || horizon <= 0 || init->count <= 0 || !init->positions || !init->masses)
            return GMPM_INVALID_ARG;
        auto r = std::unique_ptr<Request>(new (std::nothrow) Request());
        if (!r) return GMPM_OOM;
        r->desc = *d;
        r->n = init->count;
        r->pos.assign(init->positions, init->positions + 3 * init->count);
        r->mass.assign(init->masses, init->masses + init->count);
        if (init->velocities) r->vel.assign(init->velocities, init->velocities + 3 * init->count);
        if (init->material_ids) r->mat.assign(init->material_ids, init->material_ids + init->count);
        r->horizon = horizon;
        r->est_bytes = estimate_bytes(*d, init->count);
        if (opt.hbm_budget_bytes > 0 && r->est_bytes > (size_t)opt.hbm_budget_bytes) return GMPM_OOM;
        std::lock_guard<std::mutex> lk(mu);
        r->id = next_id++;
        r->t_submit = now_s() - t0;
        *id = r->id;
        queue.push_back(r->id);
        reqs[r->id] = std::move(r);
        ++st.submitted;
        return GMPM_OK;
    }

    // Admit queued requests in arrival order while the budget allows.
    void admit() {
        const double ta = now_s();
        admit_inner();
        std::lock_guard<std::mutex> lk(mu);
        st.admit_microseconds += (int64_t)((now_s() - ta) * 1e6);
    }
    void admit_inner() {
        for (;;) {
            Request* rp = nullptr;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (queue.empty()) return;
                if (opt.max_live > 0 && (int)live.size() >= opt.max_live) return;
                Request& r = *reqs[queue.front()];
                if (opt.hbm_budget_bytes > 0 && used + r.est_bytes > (size_t)opt.hbm_budget_bytes) return;
                queue.pop_front();
                rp = &r;
            }
            Request& r = *rp;
            gmpm_particle_init init{r.n, r.pos.data(), r.vel.empty() ? nullptr : r.vel.data(), r.mass.data(),
                                    r.mat.empty() ? nullptr : r.mat.data()};
            gmpm_scene* scene = nullptr;
            gmpm_status s = gmpm_scene_create(ctx, &r.desc, &init, &scene);
            const double ta = now_s() - t0;
            if (s != GMPM_OK) {
                std::lock_guard<std::mutex> lk(mu);
                r.t_admit = r.t_finish = ta;
                r.state = GMPM_REQUEST_FAILED;
                r.status = s;
                ++st.failed;
                continue;
            }
            std::vector<double>().swap(r.pos);  // the device holds the state now
            std::vector<double>().swap(r.vel);
            std::vector<double>().swap(r.mass);
            std::vector<int32_t>().swap(r.mat);
            r.bytes = std::max(r.est_bytes, scene->impl->device_bytes());
            live.push_back(&r);
            batch_stale = true;
            std::lock_guard<std::mutex> lk(mu);
            used += r.bytes;
            r.scene = scene;
            r.t_admit = ta;
            r.state = GMPM_REQUEST_RUNNING;
            ++st.admitted;
            ++st.live;
        }
    }

    // Enqueue the final reads of a request that reached its horizon, then
    // release its scene on the same stream: nothing here waits for the GPU.
    gmpm_status retire_begin(Request& r, cudaStream_t s) {
        const double tr = now_s();
        size_t need = 64;
        for (int q = 0; q < 4; ++q) {
            r.offset[q] = need;
            need += (size_t)r.n * kept_components(kKeptFields[q]) * sizeof(float);
        }
        unsigned char* buf = nullptr;
        size_t got = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            buf = pinned.acquire(need, &got);
        }
        gmpm_status e = buf ? GMPM_OK : GMPM_OOM;
        if (e == GMPM_OK) {
            r.flags = reinterpret_cast<unsigned int*>(buf);
            e = r.scene->impl->enqueue_flags(r.flags, s);
            for (int q = 0; q < 4 && e == GMPM_OK; ++q)
                e = r.scene->impl->enqueue_read(kKeptFields[q], GMPM_DTYPE_F32, GMPM_ORDER_ORIGINAL, buf + r.offset[q],
                                                s);
        }
        if (!r.ready) {
            if (!spare_events.empty()) {
                r.ready = spare_events.back();
                spare_events.pop_back();
            } else {
                cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming);
            }
        }
        cudaEventRecord(r.ready, s);
        r.scene->impl->set_release_stream(s);  // its last use was on s: free there, no device sync
        gmpm_scene_destroy(r.scene);
        {
            std::lock_guard<std::mutex> lk(mu);
            used -= std::min(used, r.bytes);
            r.scene = nullptr;
            r.results = buf;
            r.results_bytes = got;
            if (e != GMPM_OK) r.status = e;
            st.retire_microseconds += (int64_t)((now_s() - tr) * 1e6);
        }
        retiring.push_back(&r);
        return GMPM_OK;
    }

    // Complete retirements whose reads have landed (all of them when wait).
    void finish_retirements(bool wait) {
        std::vector<Request*> still;
        for (Request* r : retiring) {
            if (wait)
                cudaEventSynchronize(r->ready);
            else if (cudaEventQuery(r->ready) != cudaSuccess) {
                cudaGetLastError();
                still.push_back(r);
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            if (r->status == GMPM_OK) r->status = flags_status(*r->flags);
            r->state = r->status == GMPM_OK ? GMPM_REQUEST_DONE : GMPM_REQUEST_FAILED;
            r->t_finish = now_s() - t0;
            --st.live;
            if (r->state == GMPM_REQUEST_DONE)
                ++st.completed;
            else
                ++st.failed;
            spare_events.push_back(r->ready);
            r->ready = nullptr;
        }
        retiring.swap(still);
    }

    gmpm_status ensure_batch() {
        if (!batch_stale && batch) return GMPM_OK;
        drop_batch();
        if (live.empty()) return GMPM_OK;
        std::vector<gmpm_scene*> hs;
        for (Request* r : live) hs.push_back(r->scene);
        gmpm_batch_options o = tuned ? tuned_opt : gmpm_batch_options{};
        if (!tuned) {
            o.autotune = opt.autotune;
            o.trial_substeps = 2;
        }
        gmpm_status s = gmpm_batch_create(ctx, hs.data(), (int)hs.size(), &o, &batch);
        if (s != GMPM_OK) return s;
        if (tuned) batch_set_launch_shapes(batch, tuned_share, tuned_opt.streams);
        batch_stale = false;
        std::lock_guard<std::mutex> lk(mu);
        ++st.batches;
        return GMPM_OK;
    }

    // After a batch finished tuning, keep its choice for later batches.
    void remember_tuning() {
        if (tuned || !batch) return;
        gmpm_batch_info info;
        if (gmpm_batch_get_info(batch, &info) != GMPM_OK || !info.tuned) return;
        tuned = true;
        tuned_opt = gmpm_batch_options{};
        tuned_opt.autotune = 0;
        tuned_opt.streams = info.streams;
        // the tuned share of each size class (a class absent from the first
        // batch keeps the whole device)
        tuned_share[0] = info.sm_share_small;
        tuned_share[1] = info.sm_share_medium;
        tuned_share[2] = info.sm_share_large;
    }

    gmpm_status step(int n, cudaStream_t s) {
        if (n < 0) return GMPM_INVALID_ARG;
        SERVE_TRY(cudaSetDevice(ctx->device));
        int left = n;
        finish_retirements(false);
        if (live.empty()) admit();
        while (left > 0 && !live.empty()) {
            int64_t k = left;
            for (Request* r : live) k = std::min(k, r->horizon - r->done);
            gmpm_status e = ensure_batch();
            if (e != GMPM_OK) return e;
            const double tl = now_s();
            e = gmpm_batch_substep(batch, (int)k, s);
            if (e != GMPM_OK) return e;
            remember_tuning();
            {
                std::lock_guard<std::mutex> lk(mu);
                st.launch_microseconds += (int64_t)((now_s() - tl) * 1e6);
                for (Request* r : live) {
                    r->done += k;
                    st.particle_substeps += r->n * k;
                }
                st.substeps += k;
            }
            left -= (int)k;
            // While the GPU runs these substeps: create the scenes of waiting
            // requests (host work), then retire finished ones (waits for the GPU).
            const size_t before = live.size();
            admit();
            bool changed = live.size() != before;
            std::vector<Request*> still;
            for (Request* r : live) {
                if (r->done >= r->horizon) {
                    retire_begin(*r, s);
                    changed = true;
                } else {
                    still.push_back(r);
                }
            }
            if (changed) {
                live.swap(still);
                drop_batch();
            }
            finish_retirements(false);
        }
        // nothing left to advance: let the last retirements complete
        if (live.empty()) finish_retirements(true);
        return GMPM_OK;
    }
};

}  // namespace gmpm

struct gmpm_server {
    gmpm::Server impl;
};

extern "C" {

void gmpm_server_options_defaults(gmpm_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->hbm_budget_bytes = (int64_t)120 * 1000 * 1000 * 1000;
    o->max_live = 64;
    o->autotune = 1;
}

gmpm_status gmpm_server_create(gmpm_context* ctx, const gmpm_server_options* opt, gmpm_server** out) {
    if (!ctx || !out) return GMPM_INVALID_ARG;
    *out = nullptr;
    gmpm_server* s = new (std::nothrow) gmpm_server();
    if (!s) return GMPM_OOM;
    s->impl.ctx = ctx;
    gmpm_server_options_defaults(&s->impl.opt);
    if (opt) s->impl.opt = *opt;
    if (s->impl.opt.hbm_budget_bytes < 0 || s->impl.opt.max_live < 0) {
        delete s;
        return GMPM_INVALID_ARG;
    }
    *out = s;
    return GMPM_OK;
}

gmpm_status gmpm_server_submit(gmpm_server* s, const gmpm_scene_desc* desc, const gmpm_particle_init* init,
                               int64_t horizon, int64_t* request_id) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl.submit(desc, init, horizon, request_id);
}

gmpm_status gmpm_server_step(gmpm_server* s, int n_substeps, void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl.step(n_substeps, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_server_poll(gmpm_server* s, int64_t id, gmpm_request_status* out) {
    if (!s || !out) return GMPM_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    auto it = s->impl.reqs.find(id);
    if (it == s->impl.reqs.end()) return GMPM_INVALID_ARG;
    const gmpm::Request& r = *it->second;
    std::memset(out, 0, sizeof(*out));
    out->state = r.state;
    out->status = r.status;
    out->n_particles = r.n;
    out->substeps_done = r.done;
    out->horizon = r.horizon;
    out->submit_time = r.t_submit;
    out->admit_time = r.t_admit;
    out->finish_time = r.t_finish;
    return GMPM_OK;
}

gmpm_status gmpm_server_read(gmpm_server* s, int64_t id, int field, float* dst, size_t bytes) {
    if (!s || !dst) return GMPM_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    auto it = s->impl.reqs.find(id);
    if (it == s->impl.reqs.end() || it->second->state != GMPM_REQUEST_DONE) return GMPM_INVALID_ARG;
    const gmpm::Request& r = *it->second;
    for (int q = 0; q < 4; ++q) {
        if (gmpm::kKeptFields[q] != field) continue;
        const size_t sz = (size_t)r.n * gmpm::kept_components(field) * sizeof(float);
        if (bytes < sz || !r.results) return GMPM_INVALID_ARG;
        std::memcpy(dst, r.results + r.offset[q], sz);
        return GMPM_OK;
    }
    return GMPM_INVALID_ARG;
}

gmpm_status gmpm_server_release(gmpm_server* s, int64_t id) {
    if (!s) return GMPM_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    auto it = s->impl.reqs.find(id);
    if (it == s->impl.reqs.end()) return GMPM_INVALID_ARG;
    if (it->second->state == GMPM_REQUEST_QUEUED || it->second->state == GMPM_REQUEST_RUNNING)
        return GMPM_INVALID_ARG;
    s->impl.pinned.release(it->second->results, it->second->results_bytes);
    s->impl.reqs.erase(it);
    return GMPM_OK;
}

gmpm_status gmpm_server_get_stats(gmpm_server* s, gmpm_server_stats* out) {
    if (!s || !out) return GMPM_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    *out = s->impl.st;
    // live: counted in st under the lock
    out->queued = (int64_t)s->impl.queue.size();
    out->device_bytes_in_use = (int64_t)s->impl.used;
    return GMPM_OK;
}

gmpm_status gmpm_server_destroy(gmpm_server* s) {
    if (!s) return GMPM_INVALID_ARG;
    cudaSetDevice(s->impl.ctx->device);
    cudaDeviceSynchronize();
    delete s;
    return GMPM_OK;
}

}  // extern "C"
