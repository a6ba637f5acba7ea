// Batched stepping of independent scenes (the reference steps one scene per
// MPMSimulator::simulateStick call, Simulator.cpp:227-259).  A batch of
// uneven scenes, each with its own SPGrid, advances by one CUDA graph launch
// per substep.
//
// Scene table: the scenes whose kernels are of one kind (precision, P2G mode,
// energy models, FP64 fallback) form a group, and the group's substep is one
// launch per stage over all its scenes (launch_batch_*, kernels.h): a device
// array of the scenes' buffers and, per stage, each scene's range of CTAs.
// A graph therefore holds the same 23 kernel nodes per group whatever the
// number of scenes, and small scenes' stages fill the device together.
// Scenes that cannot join a group (the implicit phase field, whose solve
// stops on a device flag) are captured as their own launch sequences on
// parallel branches.
//
// The substep flips each scene's double-buffered particle state, so a batch
// keeps two graphs: graph k steps scene i from buffer parity0[i] ^ k, and
// replays alternate between them.  A scene stepped outside the batch changes
// its parity; the batch notices and captures again.
//
// Autotuner: the per-scene CTA ranges of the page- and slot-parallel stages
// (canon, P2G, grid, G2P) are sized for a share of the SMs per scene size
// class; the tuner times candidate shares (and, for branch scenes, the
// number of concurrent branches) on the first substeps (real substeps:
// results do not depend on launch shapes) and keeps the fastest.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <vector>

#include "kernels.h"
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

// Scenes of one kernel kind advanced by one launch per stage.
struct Group {
    int kind = 0;                      // SceneBase::batch_kind
    std::vector<int> members;          // indices into Batch::sc
    void* d_args[2] = {nullptr, nullptr};  // SceneArgs<R>[members] for graph k = 0, 1
    int32_t* d_start = nullptr;        // kBatchMaps x (members + 1) CTA range starts
    BatchPlan plan{};
    bool fp64() const { return (kind & 8) != 0; }
    size_t args_bytes() const {
        return members.size() * (fp64() ? sizeof(SceneArgs<double>) : sizeof(SceneArgs<float>));
    }
};

struct Batch {
    gmpm_context* ctx = nullptr;
    std::vector<Group> groups;
    std::vector<int> branch;           // scenes captured as their own launch sequences
    std::vector<SceneBase*> sc;
    std::vector<uint64_t> uids;
    std::vector<int> parity0;
    gmpm_batch_options opt{};
    cudaStream_t cap = nullptr;  // capture origin
    std::vector<cudaStream_t> pool;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEvent_t last = nullptr;  // after the latest graph launch
    bool launched = false;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int streams = 1;
    Candidate current{};
    std::vector<Candidate> cands;
    size_t next_cand = 0;
    bool tuned = false;
    double best_ms = 0;
    Candidate best{};
    int64_t captures = 0, substeps = 0, graph_nodes = 0, kernel_nodes = 0;
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
        // The tables may still be read by launched graphs: free them in stream
        // order after the last launch, without waiting on the host.
        if (cap) {
            if (launched) cudaStreamWaitEvent(cap, last, 0);
            for (Group& g : groups) {
                for (void*& p : g.d_args)
                    if (p) cudaFreeAsync(p, cap), p = nullptr;
                if (g.d_start) cudaFreeAsync(g.d_start, cap), g.d_start = nullptr;
            }
        }
        if (last) cudaEventDestroy(last);
        last = nullptr;
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
        // group the scenes by kernel kind; the rest go on branches
        for (int i = 0; i < n; ++i) {
            const int kind = sc[i]->batch_kind();
            if (kind < 0) {
                branch.push_back(i);
                continue;
            }
            Group* g = nullptr;
            for (Group& q : groups)
                if (q.kind == kind) g = &q;
            if (!g) {
                groups.emplace_back();
                g = &groups.back();
                g->kind = kind;
            }
            g->members.push_back(i);
        }
        const int max_streams = std::max(1, std::min<int>(n, 64));
        BATCH_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        BATCH_TRY(cudaEventCreateWithFlags(&last, cudaEventDisableTiming));
        for (Group& g : groups) {
            const size_t m = g.members.size();
            for (void*& p : g.d_args) BATCH_TRY(cudaMallocAsync(&p, g.args_bytes(), cap));
            BATCH_TRY(cudaMallocAsync(reinterpret_cast<void**>(&g.d_start), sizeof(int32_t) * kBatchMaps * (m + 1),
                                      cap));
        }
        BATCH_TRY(cudaStreamSynchronize(cap));
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
        if (!branch.empty())
            for (int st : {8, 16, 64})
                if (st <= max_streams && st != default_streams) cands.push_back(Candidate{{0, 0, 0}, st});
    }

    // Device tables of the groups for the scenes' current parities and shares
    // (outside any capture).
    gmpm_status prepare_tables() {
        if (launched && !groups.empty()) BATCH_TRY(cudaEventSynchronize(last));  // no launch still reads them
        for (Group& g : groups) {
            const int m = (int)g.members.size();
            std::vector<int32_t> start((size_t)kBatchMaps * (m + 1));
            int totals[kBatchMaps] = {};
            for (int q = 0; q < m; ++q) {
                SceneBase* s = sc[g.members[q]];
                int64_t np = 0;
                uint32_t ks = 0;
                int nb_cap = 0, ng_cap = 0;
                s->batch_sizes(&np, &ks, &nb_cap, &ng_cap);
                const int share = s->sm_share() > 0 ? std::min(s->sm_share(), ctx->num_sms) : ctx->num_sms;
                int ctas[kBatchMaps];
                batch_scene_ctas(np, ks, nb_cap, ng_cap, share, g.fp64() ? 8 : 4, ctas);
                for (int k = 0; k < kBatchMaps; ++k) {
                    start[(size_t)k * (m + 1) + q] = totals[k];
                    totals[k] += ctas[k];
                }
            }
            for (int k = 0; k < kBatchMaps; ++k) {
                start[(size_t)k * (m + 1) + m] = totals[k];
                g.plan.start[k] = g.d_start + (size_t)k * (m + 1);
                g.plan.total[k] = totals[k];
            }
            g.plan.n_scenes = m;
            g.plan.deterministic = (g.kind & 4) != 0;
            g.plan.other_models = (g.kind & 2) != 0;
            g.plan.fallback = (g.kind & 1) != 0;
            // on the batch's own stream: the copies wait for nothing else on the device
            BATCH_TRY(cudaMemcpyAsync(g.d_start, start.data(), sizeof(int32_t) * start.size(), cudaMemcpyHostToDevice,
                                      cap));
            const size_t one = g.fp64() ? sizeof(SceneArgs<double>) : sizeof(SceneArgs<float>);
            std::vector<unsigned char> host(g.args_bytes());
            for (int k = 0; k < 2; ++k) {
                for (int q = 0; q < m; ++q) {
                    const int i = g.members[q];
                    sc[i]->batch_args(parity0[i] ^ k, host.data() + (size_t)q * one);
                }
                BATCH_TRY(cudaMemcpyAsync(g.d_args[k], host.data(), host.size(), cudaMemcpyHostToDevice, cap));
                BATCH_TRY(cudaStreamSynchronize(cap));  // the host buffer is reused
            }
        }
        return GMPM_OK;
    }

    gmpm_status launch_group(const Group& g, int k, cudaStream_t s) {
        cudaError_t e;
        if (g.fp64()) {
            const auto* a = static_cast<const SceneArgs<double>*>(g.d_args[k]);
            e = launch_batch_binning<double>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_p2g<double>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_grid<double>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_g2p<double>(a, g.plan, s);
        } else {
            const auto* a = static_cast<const SceneArgs<float>*>(g.d_args[k]);
            e = launch_batch_binning<float>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_p2g<float>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_grid<float>(a, g.plan, s);
            if (e == cudaSuccess) e = launch_batch_g2p<float>(a, g.plan, s);
        }
        return e == cudaSuccess ? GMPM_OK : cuda_status(e);
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
        // the groups, one launch per stage each, on the capture stream
        for (const Group& g : groups)
            if (r == GMPM_OK) r = launch_group(g, k, cap);
        // branch scenes: largest first, spread round-robin over the branches
        std::vector<int> order(branch);
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
            std::vector<cudaGraphNode_t> list(nodes);
            kernel_nodes = 0;
            if (nodes && cudaGraphGetNodes(g, list.data(), &nodes) == cudaSuccess)
                for (cudaGraphNode_t nd : list) {
                    cudaGraphNodeType type;
                    if (cudaGraphNodeGetType(nd, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel)
                        ++kernel_nodes;
                }
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
            // the captured substeps skip the key pass (G2P keys the positions it writes)
            for (SceneBase* s : sc) {
                gmpm_status r = s->ensure_keys(cap);
                if (r != GMPM_OK) return r;
            }
            gmpm_status r = prepare_tables();
            if (r != GMPM_OK) return r;
            r = capture(0, &exec[0]);
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
            // positions written since the last substep other than by a G2P get their keys
            for (size_t i = 0; i < sc.size() && r == GMPM_OK; ++i) r = sc[i]->ensure_keys(s);
            if (r != GMPM_OK) return r;
            BATCH_TRY(cudaGraphLaunch(exec[k], s));
            BATCH_TRY(cudaEventRecord(last, s));
            launched = true;
            // a table scene's kernels are the group's launches, counted by the batch (kernel_nodes)
            for (size_t i = 0; i < sc.size(); ++i) sc[i]->commit_substeps(1, sc[i]->batch_kind() < 0);
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
        o->kernel_nodes = kernel_nodes;
        int t = 0;
        for (const Group& g : groups) t += (int)g.members.size();
        o->table_scenes = t;
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
