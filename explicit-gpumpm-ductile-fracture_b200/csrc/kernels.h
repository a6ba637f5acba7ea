// Launch entry points of the substep kernels (host side of the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "scan.cuh"
#include "state.cuh"

namespace gmpm {

struct GridDev {
    void* tile;        // [nb_cap][kP2GChannels][216] P2G page tiles (Real)
    void* nodes;       // [ng_cap][kGridChannels][64] grid results (Real)
    double* diag;      // [8] FP64 accumulators: grid mass, grid momentum xyz, ...
};

struct LaunchCfg {
    int num_sms;
    int deterministic;
};

template <typename R>
cudaError_t launch_binning(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, ScanScratch scan, Counters* cnt,
                           int num_sms, cudaStream_t stream);

// Keys + page flags only, and grid-page marking (used to size capacities).
template <typename R>
cudaError_t launch_keys(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, Counters* cnt, cudaStream_t s);
cudaError_t launch_mark_grid(BinDev bin, cudaStream_t s);

// Number of components of a gmpm_field (0 if unknown).
int field_components(int field);

// One-time per-device kernel attributes (dynamic shared memory limits).
template <typename R>
cudaError_t prepare_p2g();
template <typename R>
cudaError_t prepare_g2p();

template <typename R>
cudaError_t launch_p2g(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream);

template <typename R>
cudaError_t launch_grid(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                        cudaStream_t stream);

// sc64: the scene block in FP64 (always given; its dt drives the device
// clock).  fallback64: FP64 materials for the SVD fallback, or nullptr.
template <typename R>
cudaError_t launch_g2p(const SceneDev<R>* sc, const SceneDev<double>* sc64, const SceneDev<double>* fallback64,
                       const PState<R>& in, const PState<R>& out, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream);

// Initial constitutive evaluation (F, c, alpha, psi given; g_old = 1).
template <typename R>
cudaError_t launch_init_stress(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, int64_t n,
                               Counters* cnt, cudaStream_t stream);

// FP64 particle reductions into acc[0..7]: mass, momentum xyz, kinetic
// energy, max speed (as bits), min damage (as bits).
template <typename R>
cudaError_t launch_particle_diag(const PState<R>& st, const PAux<R>& aux, int64_t n, double* acc,
                                 cudaStream_t stream);

// Copy one field (component planes) into a packed host-layout buffer.
template <typename R>
cudaError_t launch_pack_field(const PState<R>& st, const PAux<R>& aux, int field, int dtype, int order, int64_t n,
                              void* out, cudaStream_t stream);

}  // namespace gmpm
