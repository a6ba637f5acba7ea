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
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
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
    std::map<int, std::vector<float>> results;
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
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::deque<int64_t> queue;
    std::vector<int64_t> live;
    gmpm_batch* batch = nullptr;
    bool batch_stale = true;
    bool tuned = false;
    gmpm_batch_options tuned_opt{};
    int64_t next_id = 1;
    size_t used = 0;
    gmpm_server_stats st{};
    double t0 = now_s();

    ~Server() {
        if (batch) gmpm_batch_destroy(batch);
        batch = nullptr;
        for (auto& kv : reqs)
            if (kv.second->scene) gmpm_scene_destroy(kv.second->scene);
    }

    void drop_batch() {
        if (batch) {
            gmpm_batch_info info;
            if (gmpm_batch_get_info(batch, &info) == GMPM_OK) st.capture_microseconds += (int64_t)(info.capture_seconds * 1e6);
            // only the first batch is tuned: if it ends before tuning finished,
            // later batches keep the default launch shapes
            remember_tuning();
            if (!tuned) {
                tuned = true;
                tuned_opt = gmpm_batch_options{};
            }
            gmpm_batch_destroy(batch);
        }
        batch = nullptr;
        batch_stale = true;
    }

    gmpm_status submit(const gmpm_scene_desc* d, const gmpm_particle_init* init, int64_t horizon, int64_t* id) {
        if (!d || !init || !id || horizon <= 0 || init->count <= 0 || !init->positions || !init->masses)
            return GMPM_INVALID_ARG;
        auto r = std::unique_ptr<Request>(new (std::nothrow) Request());
        if (!r) return GMPM_OOM;
        r->id = next_id++;
        r->desc = *d;
        r->n = init->count;
        r->pos.assign(init->positions, init->positions + 3 * init->count);
        r->mass.assign(init->masses, init->masses + init->count);
        if (init->velocities) r->vel.assign(init->velocities, init->velocities + 3 * init->count);
        if (init->material_ids) r->mat.assign(init->material_ids, init->material_ids + init->count);
        r->horizon = horizon;
        r->est_bytes = estimate_bytes(*d, init->count);
        r->t_submit = now_s() - t0;
        if (opt.hbm_budget_bytes > 0 && r->est_bytes > (size_t)opt.hbm_budget_bytes) return GMPM_OOM;
        *id = r->id;
        queue.push_back(r->id);
        reqs[r->id] = std::move(r);
        ++st.submitted;
        return GMPM_OK;
    }

    // Admit queued requests in arrival order while the budget allows.
    void admit() {
        while (!queue.empty()) {
            if (opt.max_live > 0 && (int)live.size() >= opt.max_live) break;
            Request& r = *reqs[queue.front()];
            if (opt.hbm_budget_bytes > 0 && used + r.est_bytes > (size_t)opt.hbm_budget_bytes) break;
            queue.pop_front();
            gmpm_particle_init init{r.n, r.pos.data(), r.vel.empty() ? nullptr : r.vel.data(), r.mass.data(),
                                    r.mat.empty() ? nullptr : r.mat.data()};
            gmpm_status s = gmpm_scene_create(ctx, &r.desc, &init, &r.scene);
            r.t_admit = now_s() - t0;
            if (s != GMPM_OK) {
                r.state = GMPM_REQUEST_FAILED;
                r.status = s;
                r.t_finish = r.t_admit;
                ++st.failed;
                continue;
            }
            r.bytes = std::max(r.est_bytes, r.scene->impl->device_bytes());
            used += r.bytes;
            r.state = GMPM_REQUEST_RUNNING;
            std::vector<double>().swap(r.pos);  // the device holds the state now
            std::vector<double>().swap(r.vel);
            std::vector<double>().swap(r.mass);
            std::vector<int32_t>().swap(r.mat);
            live.push_back(r.id);
            ++st.admitted;
            drop_batch();
        }
    }

    gmpm_status retire(Request& r, cudaStream_t s) {
        r.status = gmpm_scene_sync(r.scene);
        for (int f : kKeptFields) {
            std::vector<float>& v = r.results[f];
            v.resize((size_t)r.n * kept_components(f));
            gmpm_status e = gmpm_read_particles(r.scene, f, GMPM_DTYPE_F32, GMPM_ORDER_ORIGINAL, v.data(),
                                                v.size() * sizeof(float), s);
            if (e != GMPM_OK && r.status == GMPM_OK) r.status = e;
        }
        gmpm_scene_destroy(r.scene);
        r.scene = nullptr;
        used -= std::min(used, r.bytes);
        r.state = r.status == GMPM_OK ? GMPM_REQUEST_DONE : GMPM_REQUEST_FAILED;
        r.t_finish = now_s() - t0;
        if (r.state == GMPM_REQUEST_DONE)
            ++st.completed;
        else
            ++st.failed;
        return GMPM_OK;
    }

    gmpm_status ensure_batch() {
        if (!batch_stale && batch) return GMPM_OK;
        drop_batch();
        if (live.empty()) return GMPM_OK;
        std::vector<gmpm_scene*> hs;
        for (int64_t id : live) hs.push_back(reqs[id]->scene);
        gmpm_batch_options o = tuned ? tuned_opt : gmpm_batch_options{};
        if (!tuned) {
            o.autotune = opt.autotune;
            o.trial_substeps = 2;
        }
        gmpm_status s = gmpm_batch_create(ctx, hs.data(), (int)hs.size(), &o, &batch);
        if (s != GMPM_OK) return s;
        batch_stale = false;
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
        // one share for all sizes when the tuner chose a single one; else the largest class's
        tuned_opt.sm_share = info.sm_share_large ? info.sm_share_large
                             : info.sm_share_medium ? info.sm_share_medium
                                                    : info.sm_share_small;
    }

    gmpm_status step(int n, cudaStream_t s) {
        if (n < 0) return GMPM_INVALID_ARG;
        SERVE_TRY(cudaSetDevice(ctx->device));
        int left = n;
        admit();
        while (left > 0 && !live.empty()) {
            int64_t k = left;
            for (int64_t id : live) k = std::min(k, reqs[id]->horizon - reqs[id]->done);
            gmpm_status e = ensure_batch();
            if (e != GMPM_OK) return e;
            e = gmpm_batch_substep(batch, (int)k, s);
            if (e != GMPM_OK) return e;
            remember_tuning();
            for (int64_t id : live) {
                reqs[id]->done += k;
                st.particle_substeps += reqs[id]->n * k;
            }
            st.substeps += k;
            left -= (int)k;
            bool changed = false;
            std::vector<int64_t> still;
            for (int64_t id : live) {
                Request& r = *reqs[id];
                if (r.done >= r.horizon) {
                    retire(r, s);
                    changed = true;
                } else {
                    still.push_back(id);
                }
            }
            if (changed) {
                live.swap(still);
                drop_batch();
                admit();
            }
        }
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
    auto it = s->impl.reqs.find(id);
    if (it == s->impl.reqs.end() || it->second->state != GMPM_REQUEST_DONE) return GMPM_INVALID_ARG;
    auto f = it->second->results.find(field);
    if (f == it->second->results.end()) return GMPM_INVALID_ARG;
    if (bytes < f->second.size() * sizeof(float)) return GMPM_INVALID_ARG;
    std::memcpy(dst, f->second.data(), f->second.size() * sizeof(float));
    return GMPM_OK;
}

gmpm_status gmpm_server_release(gmpm_server* s, int64_t id) {
    if (!s) return GMPM_INVALID_ARG;
    auto it = s->impl.reqs.find(id);
    if (it == s->impl.reqs.end()) return GMPM_INVALID_ARG;
    if (it->second->state == GMPM_REQUEST_QUEUED || it->second->state == GMPM_REQUEST_RUNNING)
        return GMPM_INVALID_ARG;
    s->impl.reqs.erase(it);
    return GMPM_OK;
}

gmpm_status gmpm_server_get_stats(gmpm_server* s, gmpm_server_stats* out) {
    if (!s || !out) return GMPM_INVALID_ARG;
    *out = s->impl.st;
    gmpm_batch_info info;
    if (s->impl.batch && gmpm_batch_get_info(s->impl.batch, &info) == GMPM_OK)
        out->capture_microseconds += (int64_t)(info.capture_seconds * 1e6);
    out->live = (int64_t)s->impl.live.size();
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
