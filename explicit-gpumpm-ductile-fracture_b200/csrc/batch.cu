// Batched stepping of independent scenes: one CUDA graph per substep holds
// every scene's binning, P2G, grid update and G2P as parallel branches, so a
// batch of uneven scenes (each with its own SPGrid) is advanced by one graph
// launch instead of one launch sequence per scene (the reference steps one
// scene per MPMSimulator::simulateStick call, Simulator.cpp:227-259).
//
// The substep flips each scene's double-buffered particle state, so a batch
// keeps two graphs: graph k steps scene i from buffer parity0[i] ^ k, and
// replays alternate between them.  A scene stepped outside the batch changes
// its parity; the batch notices and captures again.
//
// Autotuner: launch shapes are sized per scene for a share of the SMs
// (small shares let small scenes' kernels run side by side).  The tuner
// times candidate shares per scene size class, and the number of concurrent
// branches, on the first substeps (real substeps: results do not depend on
// launch shapes) and keeps the fastest.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <vector>

#include "scene.h"

namespace gmpm {
namespace {

#define BATCH_TRY(expr)                                  \
    do {                                                 \
        cudaError_t e_ = (expr);                         \
        if (e_ != cudaSuccess) return cuda_status(e_);   \
    } while (0)

constexpr int64_t kSmallScene = 50000;    // particles
constexpr int64_t kMediumScene = 200000;

int size_class(int64_t n) { return n < kSmallScene ? 0 : (n < kMediumScene ? 1 : 2); }

struct Candidate {
    int share[3];  // SMs per scene by size class (0: all)
    int streams;
};

}  // namespace

struct Batch {
    gmpm_context* ctx = nullptr;
    std::vector<SceneBase*> sc;
    std::vector<uint64_t> uids;
    std::vector<int> parity0;
    gmpm_batch_options opt{};
    cudaStream_t cap = nullptr;  // capture origin
    std::vector<cudaStream_t> pool;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int streams = 1;
    Candidate current{};
    std::vector<Candidate> cands;
    size_t next_cand = 0;
    bool tuned = false;
    double best_ms = 0;
    Candidate best{};
    int64_t captures = 0, substeps = 0, graph_nodes = 0;
    double capture_s = 0;

    ~Batch() { release(); }

    void release_graphs() {
        for (auto& e : exec)
            if (e) {
                cudaGraphExecDestroy(e);
                e = nullptr;
            }
    }
    void release() {
        release_graphs();
        for (auto s : pool) cudaStreamDestroy(s);
        for (auto e : join) cudaEventDestroy(e);
        pool.clear();
        join.clear();
        if (fork) cudaEventDestroy(fork);
        if (cap) cudaStreamDestroy(cap);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        fork = t0 = t1 = nullptr;
        cap = nullptr;
    }

    gmpm_status init(gmpm_context* c, gmpm_scene* const* scenes, int n, const gmpm_batch_options* o) {
        ctx = c;
        opt = *o;
        BATCH_TRY(cudaSetDevice(ctx->device));
        for (int i = 0; i < n; ++i) {
            SceneBase* s = scenes[i]->impl;
            if (s->context() != ctx) return GMPM_INVALID_ARG;
            for (SceneBase* t : sc)
                if (t == s) return GMPM_INVALID_ARG;  // a scene appears once
            sc.push_back(s);
            uids.push_back(s->uid());
        }
        const int max_streams = std::max(1, std::min<int>(n, 64));
        BATCH_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        BATCH_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        BATCH_TRY(cudaEventCreate(&t0));
        BATCH_TRY(cudaEventCreate(&t1));
        pool.resize(max_streams);
        join.resize(max_streams);
        for (int k = 0; k < max_streams; ++k) {
            BATCH_TRY(cudaStreamCreateWithFlags(&pool[k], cudaStreamNonBlocking));
            BATCH_TRY(cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming));
        }
        const int default_streams = opt.streams > 0 ? std::min(opt.streams, max_streams) : std::min(max_streams, 32);
        current = Candidate{{opt.sm_share, opt.sm_share, opt.sm_share}, default_streams};
        if (opt.autotune) build_candidates(default_streams, max_streams);
        tuned = !opt.autotune || cands.empty();
        best = current;
        apply(current);
        return GMPM_OK;
    }

    // Coordinate search: each size class present tries shares of 1/8 .. 1 of
    // the SMs with the others at the full device, then the branch count.
    void build_candidates(int default_streams, int max_streams) {
        bool present[3] = {false, false, false};
        for (SceneBase* s : sc) present[size_class(s->particles())] = true;
        const int sms = ctx->num_sms;
        cands.push_back(Candidate{{0, 0, 0}, default_streams});
        for (int cls = 0; cls < 3; ++cls) {
            if (!present[cls]) continue;
            for (int div : {8, 4, 2}) {
                Candidate c{{0, 0, 0}, default_streams};
                c.share[cls] = std::max(1, sms / div);
                cands.push_back(c);
            }
        }
        for (int st : {8, 16, 64})
            if (st <= max_streams && st != default_streams) cands.push_back(Candidate{{0, 0, 0}, st});
    }

    void apply(const Candidate& c) {
        for (SceneBase* s : sc) s->set_sm_share(c.share[size_class(s->particles())]);
        streams = std::max(1, std::min<int>(c.streams, (int)pool.size()));
        current = c;
        release_graphs();
    }

    gmpm_status capture(int k, cudaGraphExec_t* out) {
        const auto tc = std::chrono::steady_clock::now();
        gmpm_status r = capture_graph(k, out);
        capture_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - tc).count();
        return r;
    }

    gmpm_status capture_graph(int k, cudaGraphExec_t* out) {
        BATCH_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        gmpm_status r = GMPM_OK;
        cudaError_t e = cudaEventRecord(fork, cap);
        for (int j = 0; j < streams && e == cudaSuccess; ++j) e = cudaStreamWaitEvent(pool[j], fork, 0);
        if (e != cudaSuccess) r = cuda_status(e);
        // largest scenes first, spread round-robin over the branches
        std::vector<int> order(sc.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return sc[a]->particles() > sc[b]->particles(); });
        for (size_t q = 0; q < order.size() && r == GMPM_OK; ++q) {
            const int i = order[q];
            r = sc[i]->launch_substep(pool[q % streams], parity0[i] ^ k);
        }
        for (int j = 0; j < streams && r == GMPM_OK; ++j) {
            e = cudaEventRecord(join[j], pool[j]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cap, join[j], 0);
            if (e != cudaSuccess) r = cuda_status(e);
        }
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(cap, &g);
        if (r == GMPM_OK && e != cudaSuccess) r = cuda_status(e);
        if (r == GMPM_OK) {
            size_t nodes = 0;
            cudaGraphGetNodes(g, nullptr, &nodes);
            graph_nodes = (int64_t)nodes;
            e = cudaGraphInstantiate(out, g, 0);
            if (e != cudaSuccess) r = cuda_status(e);
        }
        if (g) cudaGraphDestroy(g);
        if (r == GMPM_OK) ++captures;
        cudaGetLastError();
        return r;
    }

    // Graphs for the scenes' current parities.
    gmpm_status ensure_graphs(int* which) {
        bool ok = exec[0] && exec[1] && parity0.size() == sc.size();
        int k = 0;
        if (ok) {
            k = sc[0]->parity() ^ parity0[0];
            for (size_t i = 0; i < sc.size() && ok; ++i) ok = (sc[i]->parity() ^ parity0[i]) == k;
        }
        if (!ok) {
            release_graphs();
            parity0.resize(sc.size());
            for (size_t i = 0; i < sc.size(); ++i) parity0[i] = sc[i]->parity();
            gmpm_status r = capture(0, &exec[0]);
            if (r == GMPM_OK) r = capture(1, &exec[1]);
            if (r != GMPM_OK) {
                release_graphs();
                return r;
            }
            for (int j = 0; j < 2; ++j) BATCH_TRY(cudaGraphUpload(exec[j], cap));
            BATCH_TRY(cudaStreamSynchronize(cap));
            k = 0;
        }
        *which = k;
        return GMPM_OK;
    }

    gmpm_status replay(int n, cudaStream_t s) {
        for (int it = 0; it < n; ++it) {
            int k = 0;
            gmpm_status r = ensure_graphs(&k);
            if (r != GMPM_OK) return r;
            BATCH_TRY(cudaGraphLaunch(exec[k], s));
            for (SceneBase* q : sc) q->commit_substeps(1);
            ++substeps;
        }
        return GMPM_OK;
    }

    void set_launch_shapes(const int share[3], int nstreams) {
        Candidate c{{share[0], share[1], share[2]}, nstreams > 0 ? nstreams : current.streams};
        cands.clear();
        tuned = true;
        best = c;
        apply(c);
    }

    gmpm_status substep(int n, cudaStream_t s) {
        if (n < 0) return GMPM_INVALID_ARG;
        BATCH_TRY(cudaSetDevice(ctx->device));
        for (size_t i = 0; i < sc.size(); ++i)
            if (sc[i]->uid() != uids[i]) return GMPM_INVALID_ARG;
        const int trial = std::max(2, opt.trial_substeps + (opt.trial_substeps & 1));
        while (!tuned && n >= trial) {
            apply(cands[next_cand]);
            int k = 0;
            gmpm_status r = ensure_graphs(&k);  // capture outside the timed region
            if (r != GMPM_OK) return r;
            BATCH_TRY(cudaEventRecord(t0, s));
            r = replay(trial, s);
            if (r != GMPM_OK) return r;
            BATCH_TRY(cudaEventRecord(t1, s));
            BATCH_TRY(cudaEventSynchronize(t1));
            float ms = 0;
            BATCH_TRY(cudaEventElapsedTime(&ms, t0, t1));
            const double per = ms / trial;
            if (next_cand == 0 || per < best_ms) {
                best_ms = per;
                best = cands[next_cand];
            }
            n -= trial;
            if (++next_cand == cands.size()) {
                tuned = true;
                apply(best);
            }
        }
        return replay(n, s);
    }

    void info(gmpm_batch_info* o) const {
        std::memset(o, 0, sizeof(*o));
        o->n_scenes = (int32_t)sc.size();
        o->streams = streams;
        o->tuned = tuned ? 1 : 0;
        o->n_candidates = (int32_t)cands.size();
        o->graph_nodes = graph_nodes;
        o->captures = captures;
        o->substeps = substeps;
        o->best_ms_per_substep = best_ms;
        o->sm_share_small = current.share[0];
        o->sm_share_medium = current.share[1];
        o->sm_share_large = current.share[2];
        o->capture_seconds = capture_s;
    }
};

}  // namespace gmpm

struct gmpm_batch {
    gmpm::Batch impl;
};

extern "C" {

void gmpm_batch_options_defaults(gmpm_batch_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->autotune = 1;
    o->trial_substeps = 2;
    o->streams = 0;
    o->sm_share = 0;
}

gmpm_status gmpm_batch_create(gmpm_context* ctx, gmpm_scene* const* scenes, int n_scenes,
                              const gmpm_batch_options* opt, gmpm_batch** out) {
    if (!ctx || !out || n_scenes <= 0 || !scenes) return GMPM_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < n_scenes; ++i)
        if (!scenes[i] || !scenes[i]->impl) return GMPM_INVALID_ARG;
    gmpm_batch_options o;
    gmpm_batch_options_defaults(&o);
    if (opt) o = *opt;
    if (o.trial_substeps < 0 || o.streams < 0 || o.sm_share < 0) return GMPM_INVALID_ARG;
    gmpm_batch* b = new (std::nothrow) gmpm_batch();
    if (!b) return GMPM_OOM;
    gmpm_status r = b->impl.init(ctx, scenes, n_scenes, &o);
    if (r != GMPM_OK) {
        delete b;
        cudaGetLastError();
        return r;
    }
    *out = b;
    return GMPM_OK;
}

gmpm_status gmpm_batch_substep(gmpm_batch* b, int n_substeps, void* stream) {
    if (!b) return GMPM_INVALID_ARG;
    return b->impl.substep(n_substeps, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_batch_get_info(gmpm_batch* b, gmpm_batch_info* out) {
    if (!b || !out) return GMPM_INVALID_ARG;
    b->impl.info(out);
    return GMPM_OK;
}

gmpm_status gmpm_batch_destroy(gmpm_batch* b) {
    if (!b) return GMPM_INVALID_ARG;
    cudaSetDevice(b->impl.ctx->device);
    cudaDeviceSynchronize();  // graph launches may still be in flight on the caller's stream
    delete b;
    return GMPM_OK;
}

}  // extern "C"

namespace gmpm {
// Destroy a batch whose graph launches may still run: executable graphs,
// streams and events may be destroyed with work in flight (the driver
// releases them when it completes), so no synchronisation is needed.  The
// scenes' memory is untouched.
void batch_destroy_deferred(gmpm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->impl.ctx->device);
    delete b;
}

void batch_set_launch_shapes(gmpm_batch* b, const int share[3], int streams) {
    if (b) b->impl.set_launch_shapes(share, streams);
}
}  // namespace gmpm

extern "C" {

}  // extern "C"
