// Launch entry points of the substep kernels (host side of the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "scan.cuh"
#include "state.cuh"

namespace gmpm {

// Device scalars of the implicit phase-field solve.
struct PcgScalars {
    double rho_old, alpha, rate, norm;
    int done;        // converged, blew up or capped: later kernels of the solve return at once
    int blowup;      // rho_old == 0: the reference sets x = 1e20 everywhere
    int iterations;  // iterations of the current solve
    int pad;
};

// Vectors of the implicit phase-field solve, FP64 over the grid nodes
// (ng_cap * 64, in grid-page order), and the per-particle col vectors.
struct PcgDev {
    double* x;
    double* r;
    double* mr;
    double* s;
    double* q;
    double* d;     // Jacobi diagonal sum_p V w (FP M + 1/dt)
    double* cg;    // c_grid = sum w c / sum w
    uint8_t* tag;  // node touched by a particle
    double* col;   // [3][n] 4 L0^2 V grad s at the particles (sorted order)
    double* part;  // [3][nparts_cap] partial sums over runs of 128 entries
    PcgScalars* scal;
    int64_t nparts_cap;
    int64_t n;     // particles (col stride)
};

struct GridDev {
    void* tile;        // [nb_cap][kP2GChannels][216] P2G page tiles (Real); also the solve's FP64 node tiles
    void* nodes;       // [ng_cap][kGridChannels][64] grid results (Real)
    double* diag;      // [8] FP64 accumulators: grid mass, grid momentum xyz, ...
    PcgDev pcg;        // implicit phase field only (null pointers otherwise)
};

struct LaunchCfg {
    int num_sms;
    int deterministic;
    int pcg_max_combine;   // implicit phase field settings
    double pcg_mobility;
    double pcg_tolerance;
    int other_models;      // a material uses an energy model other than von Mises
};

// keys_ready: bin.keys and bin.page_flag already hold the keys and pages of
// st's positions (written by the G2P that produced them), so the key pass is
// skipped and the page flags are cleared after their last use, for the next
// G2P to set.  Otherwise the key pass runs and the flags stay set.
template <typename R>
cudaError_t launch_binning(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, ScanScratch scan, Counters* cnt,
                           int num_sms, cudaStream_t stream, bool keys_ready = false);
// Kernels launched by launch_binning without / with keys_ready.
constexpr int kBinningKernels = 17;
constexpr int kBinningKernelsKeysReady = 16;

// Keys + page flags only, and grid-page marking (used to size capacities).
template <typename R>
cudaError_t launch_keys(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, Counters* cnt, cudaStream_t s);
cudaError_t launch_mark_grid(BinDev bin, cudaStream_t s);
// The counting-sort passes of the binning (also used by the allocation-free entry point).
cudaError_t launch_bin_hist(int64_t n, const uint32_t* keys, const int32_t* page_rank, int32_t* cell_count, int nb_cap,
                            cudaStream_t s);
cudaError_t launch_bin_scatter(int64_t n, const uint32_t* keys, const int32_t* page_rank, const int32_t* cell_start,
                               int32_t* fill, int32_t* perm, uint32_t* keys_sorted, int nb_cap, cudaStream_t s);
cudaError_t launch_bin_canon(BinDev bin, Counters* cnt, int num_sms, cudaStream_t s);

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

// Implicit phase field (pcg.cu): init after the grid kernel, one CG iteration
// per call (kernels return at once after convergence), finish before G2P.
template <typename R>
cudaError_t launch_pcg_init(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                            cudaStream_t stream);
template <typename R>
cudaError_t launch_pcg_iteration(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin,
                                 GridDev grid, Counters* cnt, LaunchCfg cfg, cudaStream_t stream);
template <typename R>
cudaError_t launch_pcg_finish(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                              cudaStream_t stream);
constexpr int kPcgInitKernels = 2, kPcgIterationKernels = 7, kPcgFinishKernels = 1;

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

// ---- batched launches: one launch per stage over many scenes ------------------
// A batch of scenes of one kind (precision, P2G mode, energy models, FP64
// fallback) advances with one launch per stage of the substep.  Every stage
// splits its launch into per-scene CTA ranges (BatchPlan); a CTA finds its
// scene by a search over its stage's range starts and runs the stage's body
// for that scene with its place in the scene's range (VB, common.cuh).

// One scene's buffers as the stages of a batched substep see them, for the
// parity that reads state `in` and writes `out`.
template <typename R>
struct SceneArgs {
    const SceneDev<R>* sc;
    const SceneDev<double>* sc64;
    PState<R> in, out;
    PAux<R> aux;
    BinDev bin;
    GridDev grid;
    Counters* cnt;
    ScanScratch scan;
};

// The scene of this CTA in a batched launch, with its SceneArgs copied into
// `sa` (a __shared__ variable of the kernel).  A one-scene kernel reads its
// buffers' addresses from the constant bank where it uses them; a batched
// body given references into A keeps them live in registers across its
// loops.  Reading them from `sa` removes the grid body's spills.  The P2G and
// G2P bodies spill as much or more with the copy, and read A.
template <typename R>
__device__ __forceinline__ const SceneArgs<R>& batch_scene_args(const SceneArgs<R>* __restrict__ A,
                                                                const int32_t* __restrict__ start, int ns, VB& vb,
                                                                SceneArgs<R>& sa) {
    static_assert(sizeof(SceneArgs<R>) % 4 == 0, "copied in 4-byte words");
    const int s = scene_of_block(start, ns, vb);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&A[s]);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
    for (int w = (int)threadIdx.x; w < (int)(sizeof(SceneArgs<R>) / 4); w += (int)blockDim.x) dst[w] = src[w];
    __syncthreads();
    return sa;
}

// Per-scene CTA ranges of the stages (device arrays of n_scenes + 1 starts).
enum BatchMap : int {
    BM_ZERO_FLAGS = 0,  // key_space bytes in 4 KiB pieces
    BM_PARTICLES,       // particles, 4 per thread (histogram, scatter)
    BM_KEYSPACE,        // one thread per page key (grid marking, compaction)
    BM_KEY_TILES,       // scan tiles of the key space
    BM_LINKS,           // page links
    BM_ZERO_CELLS,      // cell counters (and page flags) in 4 KiB pieces
    BM_CELL_TILES,      // scan tiles of the cell counters
    BM_CANON,
    BM_P2G,
    BM_GRID,
    BM_G2P,
    BM_ONE,             // one CTA per scene (scan of the tile sums, clock, diagnostics reset)
    kBatchMaps
};

struct BatchPlan {
    int n_scenes;
    const int32_t* start[kBatchMaps];  // device
    int total[kBatchMaps];             // CTAs of each launch
    int deterministic;                 // P2G's fixed-order mode
    int other_models;                  // a material uses an energy model other than von Mises
    int fallback;                      // FP32 with the FP64 SVD fallback
};

// Host-side CTA counts of one scene per map (the same shapes as its one-scene
// launches; canon, P2G, grid and G2P sized for `sms` SMs).
void batch_scene_ctas(int64_t n, uint32_t key_space, int nb_cap, int ng_cap, int sms, int real_bytes,
                      int ctas[kBatchMaps]);

// The batch's scenes enter with their keys and page flags set by the G2P (or
// key pass) that wrote their positions, as launch_binning with keys_ready.
template <typename R>
cudaError_t launch_batch_binning(const SceneArgs<R>* args, const BatchPlan& plan, cudaStream_t s);
template <typename R>
cudaError_t launch_batch_p2g(const SceneArgs<R>* args, const BatchPlan& plan, cudaStream_t s);
template <typename R>
cudaError_t launch_batch_grid(const SceneArgs<R>* args, const BatchPlan& plan, cudaStream_t s);
template <typename R>
cudaError_t launch_batch_g2p(const SceneArgs<R>* args, const BatchPlan& plan, cudaStream_t s);
constexpr int kBatchLaunchesPerSubstep = 23;

}  // namespace gmpm
