// Host-side scene interface shared by the C-ABI (api.cu), batched stepping
// (batch.cu) and the serving loop (serve.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gmpm.h"

struct gmpm_context {
    int device;
    int num_sms;
    cudaDeviceProp prop;
};

namespace gmpm {

gmpm_status cuda_status(cudaError_t e);

// Common scene interface, implemented per precision (Scene<R> in api.cu).
struct SceneBase {
    virtual ~SceneBase() {}
    virtual gmpm_status substep(int n, cudaStream_t s) = 0;
    virtual gmpm_status substep_timed(int n, cudaStream_t s, gmpm_stage_times* out) = 0;
    virtual gmpm_status rebin(cudaStream_t s) = 0;
    virtual gmpm_status read_particles(int field, int dtype, int order, void* dst, size_t bytes, cudaStream_t s) = 0;
    // Read overlapped with later work: packed on s, copied on the scene's copy
    // stream; complete after reads_wait.
    virtual gmpm_status read_particles_async(int field, int dtype, int order, void* dst, size_t bytes,
                                             cudaStream_t s) = 0;
    virtual gmpm_status reads_wait() = 0;
    virtual gmpm_status read_binning(int array, void* dst, size_t bytes) = 0;
    virtual gmpm_status diagnostics(gmpm_diag* out) = 0;
    virtual gmpm_status sync() = 0;
    virtual gmpm_status set_dt(double dt, cudaStream_t s) = 0;
    virtual gmpm_status set_velocity_conditions(const gmpm_slab_bc* slabs, int ns, const gmpm_sphere_bc* spheres,
                                                int nsp, cudaStream_t s) = 0;

    // Batched stepping.  launch_substep issues one substep's kernels for the
    // given state buffer without touching host bookkeeping, so it can be
    // captured into a CUDA graph; commit_substeps records n substeps that
    // were launched that way (buffer flips, launch counts).
    virtual uint64_t uid() const = 0;
    virtual gmpm_context* context() const = 0;
    virtual int64_t particles() const = 0;
    virtual size_t device_bytes() const = 0;
    virtual int parity() const = 0;
    virtual int kernels_per_substep() const = 0;
    virtual gmpm_status launch_substep(cudaStream_t s, int parity) = 0;
    // A key pass over the current positions on s, unless the last writer of
    // the positions (a G2P or an earlier key pass) left their keys in place;
    // substeps captured afterwards skip their key pass.
    virtual gmpm_status ensure_keys(cudaStream_t s) = 0;
    // own_launches: the substeps ran the scene's own kernels (a branch or the
    // plain path), not a batch's launches over many scenes.
    virtual void commit_substeps(int n, bool own_launches = true) = 0;
    // Launch shapes are sized for this many SMs (0: the whole device).
    virtual void set_sm_share(int sms) = 0;
    virtual int sm_share() const = 0;
    // One launch per stage over many scenes (kernels.h, BatchPlan): the kind of
    // the scene's kernels (precision, P2G mode, energy models, FP64 fallback;
    // -1 if the scene cannot join, as with the implicit phase field), its
    // buffers for a parity as a SceneArgs<R> (into out), and the sizes that
    // set its CTA ranges.
    virtual int batch_kind() const = 0;
    virtual void batch_args(int parity, void* out) const = 0;
    virtual void batch_sizes(int64_t* n, uint32_t* key_space, int* nb_cap, int* ng_cap) const = 0;

    // Checkpoint of the particle state and clock (gmpm_scene_save).
    virtual gmpm_status save(const char* path) = 0;

    // Serving: status flags read on a stream (no device synchronisation), and
    // release of the scene's memory on a stream after its last use there.
    virtual gmpm_status status_on_stream(cudaStream_t s) = 0;
    virtual void set_release_stream(cudaStream_t s) = 0;
    // Enqueue (no wait) a read of one field into pinned or device memory, and
    // of the status flags into pinned memory.
    virtual gmpm_status enqueue_read(int field, int dtype, int order, void* dst, cudaStream_t s) = 0;
    virtual gmpm_status enqueue_flags(unsigned int* dst, cudaStream_t s) = 0;
};

// Destroy a batch without synchronising the device (its graphs may still run).
void batch_destroy_deferred(gmpm_batch* b);
// Fix a batch's launch shapes without tuning: SMs per scene by size class
// (< 50k, < 200k, larger particles; 0: all) and the number of branches.
void batch_set_launch_shapes(gmpm_batch* b, const int share[3], int streams);

// Status of a set of device flags (GMPM_FLAG_*).
gmpm_status flags_status(unsigned int flags);

}  // namespace gmpm

struct gmpm_scene {
    gmpm::SceneBase* impl;
};
