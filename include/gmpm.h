/*
 * gmpm.h — C-ABI of the B200-native explicit MPM ductile-fracture substep.
 *
 * The library runs the explicit APIC-MPM substep of
 * KemengHuang/Explicit-GPUMPM-Ductile-Fracture on a sparse paged grid (SPGrid:
 * 4x4x4-node pages addressed by Morton-interleaved page keys):
 *   particle binning by page/cell key  ->  P2G  ->  grid update (gravity,
 *   walls, velocity conditions, explicit phase-field evolution)  ->  G2P with
 *   the C-matrix and F update, 3x3 QR/Givens SVD, Hencky plastic return
 *   mapping with hardening and the plastic-strain-driven damage update.
 *
 * Every entry point returns a gmpm_status; nothing calls exit().  The library
 * owns all device memory; the caller owns host buffers.  One host thread per
 * context.  Stream arguments are `cudaStream_t` passed as `void*` (NULL = the
 * legacy default stream).
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root).
 */
#ifndef GMPM_H
#define GMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GMPM_ABI_VERSION 1

/* Status codes.  Replaces CUDA_SAFE_CALL's print-and-exit(0)
 * (GPU_MPM/cuda_tools.h:25-36) and unchecked kernel launches. */
typedef enum gmpm_status {
    GMPM_OK = 0,
    GMPM_INVALID_ARG = 1,
    GMPM_OOM = 2,
    GMPM_TABLE_OVERFLOW = 3,   /* block/page capacity exceeded (reference: unbounded hash probes) */
    GMPM_NONFINITE = 4,        /* non-finite particle state detected */
    GMPM_OUT_OF_DOMAIN = 5,    /* particle stencil left the grid (reference quirk: negative base node) */
    GMPM_CUDA_ERROR = 6,
    GMPM_NOT_SUPPORTED = 7,
    GMPM_NO_DEVICE = 8,
    GMPM_IO_ERROR = 9          /* a checkpoint file could not be written, read or recognised */
} gmpm_status;

/* Device-side status flags accumulated during substeps (gmpm_diagnostics.flags). */
#define GMPM_FLAG_OUT_OF_DOMAIN   0x1u
#define GMPM_FLAG_NONFINITE       0x2u
#define GMPM_FLAG_SVD_NOCONVERGE  0x4u
#define GMPM_FLAG_TABLE_OVERFLOW  0x8u   /* page capacity exceeded, or a cell above 6144 particles
                                            (that cell then keeps a non-canonical order) */
#define GMPM_FLAG_COPY_TIMEOUT    0x10u  /* an asynchronous copy did not complete within the kernel's bounded
                                            wait; the kernel stopped early (reported as GMPM_CUDA_ERROR) */

typedef enum gmpm_precision {
    GMPM_PRECISION_FP32 = 0,          /* FP32 state and arithmetic */
    GMPM_PRECISION_FP64 = 1,          /* FP64 everywhere (reference precision, Setting.h:3-5) */
    GMPM_PRECISION_FP32_FP64SVD = 2   /* FP32 bulk; FP64 SVD + return map when sigma_min/sigma_max < svd_fallback_ratio */
} gmpm_precision;

typedef enum gmpm_hardening {
    GMPM_HARDENING_EXPONENTIAL = 0,   /* reference R(alpha) (ExplicitTimeIntegrator.cu:64-68) */
    GMPM_HARDENING_LINEAR = 1         /* R(alpha) = yield + H * alpha */
} gmpm_hardening;

/* Energy model of a material: the reference's compile-time Energy_Model
 * (Setting.h:38), selectable per material here. */
typedef enum gmpm_energy_model {
    GMPM_ENERGY_VON_MISES_FRACTURE = 0,  /* Energy_Model 2: Hencky von Mises plasticity with hardening and
                                            phase-field fracture (applyVonMises,
                                            ExplicitTimeIntegrator.cu:132-370) */
    GMPM_ENERGY_FIXED_COROTATED = 1,     /* Energy_Model 0: elastic fixed-corotated, no fracture driving
                                            (computeContributionFixedCorotated, :22-47) */
    GMPM_ENERGY_NEO_HOOKEAN_FRACTURE = 2 /* Energy_Model 1: elastic Neo-Hookean with the tension/compression
                                            split and phase-field fracture driving; G_c = 3 and L0 = dx/2 as
                                            hard-coded there (computeContributionNeoHookean, :372-446) */
} gmpm_energy_model;

typedef enum gmpm_phase_field {
    GMPM_PHASE_FIELD_OFF = 0,
    GMPM_PHASE_FIELD_EXPLICIT = 1,    /* explicit diffusion, pointwise-implicit reaction */
    GMPM_PHASE_FIELD_IMPLICIT = 2     /* the reference's Jacobi-preconditioned CG solve of
                                         (D + M K) c = M_L (c_grid/dt + M) each substep
                                         (ExplicitTimeIntegrator.cu:909-972) */
} gmpm_phase_field;

/* Material and fracture constants.  Replaces ElasticMaterial
 * (GPU_MPM/Materials.h:15-23, Materials.cpp:4-13) and the constants hard-coded
 * in applyVonMises (GPU_MPM/ExplicitTimeIntegrator.cu:188-194,320-335). */
typedef struct gmpm_material {
    double youngs_modulus;     /* E */
    double poisson_ratio;      /* nu */
    double density;            /* rho (informational; particle masses are explicit) */
    double yield_stress;       /* reference 800 */
    int32_t hardening_law;     /* gmpm_hardening */
    int32_t energy_model;      /* gmpm_energy_model; 0 (von Mises with fracture) by default */
    double hardening;          /* exponential rate h (reference 3) or linear modulus H */
    double alpha_cap;          /* alpha_c, reference 1 */
    double dlambda_cap;        /* reference 100 */
    double strain_cap;         /* Hencky strain clamp, reference 3 */
    double psi_cap;            /* psi+ history accepted below this, reference 1e6 */
    double fracture_energy;    /* G_c0, reference 3 */
    double softening_onset;    /* ps, softening when alpha/2 > ps; reference 0.01 */
    double residual_fracture;  /* residual G_c fraction, reference 0.1 */
    double theta;              /* degradation floor, reference 0.0001f (float) */
    double length_scale;       /* L0, reference 0.5*dx */
    double mobility;           /* M, reference 50 (Materials.cpp:13) */
} gmpm_material;

/* Velocity condition on nodes inside an axis-aligned slab lo <= x[axis] <= hi. */
typedef struct gmpm_slab_bc {
    int32_t axis;
    int32_t _pad0;
    double lo, hi;
    double velocity[3];
} gmpm_slab_bc;

/* Rigid sphere moving at constant velocity; nodes inside take its velocity
 * (generalises PullGrid_kernal, GPU_MPM/TimeIntegrator.cu:169-261). */
typedef struct gmpm_sphere_bc {
    double center[3];          /* at t = 0 */
    double radius;
    double velocity[3];
} gmpm_sphere_bc;

#define GMPM_MAX_SLAB_BCS 4
#define GMPM_MAX_MATERIALS 8
#define GMPM_MAX_SPHERE_BCS 2

typedef struct gmpm_scene_desc {
    double dx;                 /* grid spacing (Setting.h:14) */
    int32_t grid_res[3];       /* nodes per axis; domain [0, grid_res*dx) */
    int32_t _pad0;
    double dt;                 /* fixed substep (Simulator.cpp:172,213) */
    double gravity[3];         /* reference: (0,-10,0) hard-coded (TimeIntegrator.cu:100) */
    double particle_volume;    /* V0 (Simulator.cpp:181) */
    int32_t n_materials;       /* 1..GMPM_MAX_MATERIALS; particles select one by material id */
    int32_t _pad1;
    gmpm_material materials[GMPM_MAX_MATERIALS];
    int32_t wall_bc;           /* 1 = sticky walls (collideWithGround, TimeIntegrator.cu:117-165) */
    int32_t wall_layers;       /* nodes i <= wall_layers or i > res - wall_layers; reference 4 */
    int32_t n_slab_bcs;
    int32_t n_sphere_bcs;
    gmpm_slab_bc slabs[GMPM_MAX_SLAB_BCS];
    gmpm_sphere_bc spheres[GMPM_MAX_SPHERE_BCS];
    int32_t precision;         /* gmpm_precision */
    int32_t phase_field;       /* gmpm_phase_field */
    int32_t deterministic;     /* 1 = fixed-order P2G (bitwise reproducible), 0 = atomic fast mode */
    int32_t block_capacity;    /* max active pages; 0 = derive from the particle count */
    double svd_fallback_ratio; /* sigma_min/sigma_max threshold for the FP64 fallback (1e-3) */
    int32_t adaptive_dt;       /* 1: each substep's dt = min(dt, cfl_number dx / max |v_p|), computed on the
                                  device from the previous G2P's velocities (MPMSimulator::computeDt,
                                  Simulator.cpp:200-225, without its host read); dt is then the upper bound */
    int32_t _pad2;
    double cfl_number;         /* 0.3f as in computeDt (default) */
    int32_t pcg_max_iterations; /* implicit phase field: iteration cap (100, ExplicitTimeIntegrator.cu:925) */
    int32_t pcg_max_combine;   /* 1: dot products combine per-128-entry partial sums with max, as the
                                  reference's getDotProduct does (quirk); 0: true sums (default) */
    double pcg_tolerance;      /* stop when max |r| < tolerance (1e-6, :926) */
} gmpm_scene_desc;

/* Initial particle state.  Replaces the h_pos/h_vel/h_mass arrays handed to
 * Particles::initialize (GPU_MPM/Particles.cuh:12, Particles.cpp:8-31).
 * positions/velocities are count x 3 (xyz interleaved), masses count.
 * count must be below 2^28 (the material id shares the id word). */
typedef struct gmpm_particle_init {
    int64_t count;
    const double* positions;
    const double* velocities;  /* may be NULL (zero) */
    const double* masses;
    const int32_t* material_ids; /* may be NULL (all 0); each < n_materials */
} gmpm_particle_init;

/* Particle fields for gmpm_read_particles. Matrices are 3x3 column-major
 * (element (r,c) at r + 3c), as the reference stores d_F / d_B planes. */
typedef enum gmpm_field {
    GMPM_FIELD_POSITION = 0,   /* 3 */
    GMPM_FIELD_VELOCITY = 1,   /* 3 */
    GMPM_FIELD_F = 2,          /* 9 */
    GMPM_FIELD_B = 3,          /* 9, APIC affine matrix */
    GMPM_FIELD_DAMAGE = 4,     /* 1, phase field c (1 = intact) */
    GMPM_FIELD_ALPHA = 5,      /* 1, equivalent plastic strain */
    GMPM_FIELD_PSI_MAX = 6,    /* 1, tensile energy history */
    GMPM_FIELD_STRESS = 7,     /* 6, V0*P*F^T symmetric: xx yy zz xy xz yz */
    GMPM_FIELD_VOLUME = 8,     /* 1, V0*det F */
    GMPM_FIELD_FP = 9,         /* 1, fracture driving coefficient */
    GMPM_FIELD_PF_FLUX = 10,   /* 3, 4 L0^2 V grad(c) carried to the next P2G */
    GMPM_FIELD_MASS = 11,      /* 1 */
    GMPM_FIELD_ID = 12,        /* 1, original particle index (int32) */
    GMPM_FIELD_COUNT = 13
} gmpm_field;

typedef enum gmpm_dtype {
    GMPM_DTYPE_F64 = 0,
    GMPM_DTYPE_F32 = 1,
    GMPM_DTYPE_I32 = 2
} gmpm_dtype;

typedef enum gmpm_order {
    GMPM_ORDER_INTERNAL = 0,   /* current sorted order (what Attribs_Back_Host copies) */
    GMPM_ORDER_ORIGINAL = 1    /* original particle index order */
} gmpm_order;

/* Binning arrays for gmpm_read_binning (bit-exact parity with the oracle). */
typedef enum gmpm_binning_array {
    GMPM_BIN_COUNTS = 0,       /* int64[4]: n_particles, n_blocks, n_grid_blocks, key_space */
    GMPM_BIN_PERM = 1,         /* int32[n]: new slot -> previous slot (d_indexTrans) */
    GMPM_BIN_KEYS = 2,         /* uint32[n]: (page_key << 6) | cell, sorted */
    GMPM_BIN_BLOCK_KEYS = 3,   /* uint32[n_blocks]: active page keys, ascending */
    GMPM_BIN_BLOCK_START = 4,  /* int32[n_blocks + 1]: particle range per page */
    GMPM_BIN_CELL_START = 5,   /* int32[n_blocks * 64 + 1]: particle range per cell */
    GMPM_BIN_GRID_KEYS = 6,    /* uint32[n_grid_blocks]: pages incl. + neighbours, ascending */
    GMPM_BIN_ADJ = 7,          /* int32[n_blocks * 8]: grid-block index of page + (i,j,k), slot 4i+2j+k */
    GMPM_BIN_COUNT = 8
} gmpm_binning_array;

typedef struct gmpm_diag {
    double particle_mass;      /* sum m_p */
    double particle_momentum[3];
    double grid_mass;          /* sum over nodes after the last P2G */
    double grid_momentum[3];   /* sum m_i v_i after the last P2G (incl. dt*f) */
    double kinetic_energy;
    double max_speed;          /* for CFL dt (Simulator.cpp:200-225) */
    double min_damage;
    double time;               /* simulated time */
    int64_t substeps;
    int64_t n_particles;
    int32_t n_blocks;
    int32_t n_grid_blocks;
    uint32_t flags;            /* GMPM_FLAG_* accumulated since creation */
    int32_t _pad0;
    int64_t kernel_launches;   /* kernels this scene launched since creation */
    double dt;                 /* time step of the next substep */
    int32_t pcg_iterations;    /* implicit phase field: CG iterations of the last substep */
    int32_t _pad1;
} gmpm_diag;

/* Per-stage device time of gmpm_substep_timed, summed over its substeps
 * (CUDA events on the launching stream). */
typedef struct gmpm_stage_times {
    double bin_ms;             /* binning: keys, page tables, counting sort */
    double p2g_ms;
    double grid_ms;
    double g2p_ms;             /* G2P + constitutive update */
    double total_ms;
    int64_t substeps;
} gmpm_stage_times;

typedef struct gmpm_context gmpm_context;
typedef struct gmpm_scene gmpm_scene;

/* ---- context / scene lifetime -------------------------------------------- */

/* Replaces cudaSetDevice(0) in init_cuda (GPU_MPM/gl_main.cpp:31-37). */
gmpm_status gmpm_context_create(int device, gmpm_context** out);
gmpm_status gmpm_context_destroy(gmpm_context* ctx);

/* Reference-default scene: the constants of Setting.h and applyVonMises with a
 * caller-chosen grid.  Replaces the compile-time configuration
 * (GPU_MPM/Setting.h:3-38) and the material of MPMSimulator::build
 * (GPU_MPM/Simulator.cpp:114-116). */
gmpm_status gmpm_scene_desc_reference_defaults(gmpm_scene_desc* desc, double dx, int res_x, int res_y, int res_z);

/* Replaces MPMSimulator::build (GPU_MPM/Simulator.cpp:76-198): allocation
 * (MallocDeviceMEM :16-31, Particles_Malloc_MEM, SPGrid_MEM_Malloc,
 * Transformer_Malloc_MEM), Particles::initialize (Particles.cpp:8-31,
 * Particle_kernal.cu:441-481), F = I and B = 0 (buildIntegrator :67-74).
 * Also evaluates the initial stress so the first substep can start at P2G. */
gmpm_status gmpm_scene_create(gmpm_context* ctx, const gmpm_scene_desc* desc,
                              const gmpm_particle_init* init, gmpm_scene** out);
gmpm_status gmpm_scene_destroy(gmpm_scene* scene);

/* ---- stepping ------------------------------------------------------------- */

/* n substeps of fixed dt.  Replaces ExplicitTimeIntegrator::integrate
 * (GPU_MPM/ExplicitTimeIntegrator.cu:881-994) including
 * DomainTransformer::rebuild (Transformer.cpp:71-82) and Particles::reorder
 * (Particle_kernal.cu:544-573).  Asynchronous on `stream`; no host syncs. */
gmpm_status gmpm_substep(gmpm_scene* scene, int n, void* stream);

/* gmpm_substep with CUDA events between the stages; waits for completion and
 * returns the device time of each stage.  Replaces the cudaEvent timers of
 * ExplicitTimeIntegrator::integrate (ExplicitTimeIntegrator.cu:884-994) that
 * report preprocess and simulation time. */
gmpm_status gmpm_substep_timed(gmpm_scene* scene, int n, void* stream, gmpm_stage_times* out);

/* Change the substep size (asynchronous on `stream`).  Serves the CFL time
 * step of MPMSimulator::computeDt (GPU_MPM/Simulator.cpp:200-225), which the
 * reference passes to integrate() every frame. */
gmpm_status gmpm_set_dt(gmpm_scene* scene, double dt, void* stream);

/* Replace the scene's velocity conditions (slabs and moving spheres) from
 * host memory, asynchronously on `stream` (pass pinned memory to keep the
 * copy asynchronous).  Counts must not exceed GMPM_MAX_SLAB_BCS /
 * GMPM_MAX_SPHERE_BCS.  Generalises the time-dependent spheres of
 * PullGrid_kernal (GPU_MPM/TimeIntegrator.cu:169-261), whose motion the
 * reference hard-codes in the kernel. */
gmpm_status gmpm_set_velocity_conditions(gmpm_scene* scene, const gmpm_slab_bc* slabs, int n_slabs,
                                         const gmpm_sphere_bc* spheres, int n_spheres, void* stream);

/* Binning alone on the current positions (sort + page tables).  Replaces
 * Particles::sort_by_offsets (Particle_kernal.cu:484-542) followed by
 * DomainTransformer::rebuild (Transformer.cpp:71-82). */
gmpm_status gmpm_rebin(gmpm_scene* scene, void* stream);

/* Wait for all work queued on the scene's streams and report accumulated flags
 * as a status (OUT_OF_DOMAIN / NONFINITE / TABLE_OVERFLOW). */
gmpm_status gmpm_scene_sync(gmpm_scene* scene);

/* ---- readback ------------------------------------------------------------- */

/* Copy one particle field to `dst` (host or device pointer, `bytes` capacity).
 * Replaces Particles::Attribs_Back_Host (GPU_MPM/Particles.cpp:33-52). */
gmpm_status gmpm_read_particles(gmpm_scene* scene, int field, int dtype, int order,
                                void* dst, size_t bytes, void* stream);

/* Copy one binning array (gmpm_binning_array) to host memory.  Exposes what
 * the reference keeps in Particles/DomainTransformer device members
 * (d_indexTrans, cell_id, d_page2particle, d_cell2particle, d_adjPage:
 * GPU_MPM/Particles.cuh:26-44, Transformer.cuh:35-50). */
/* Overlapped read for frame loops (Attribs_Back_Host, Particles.cpp:33-52, without the stall): the
 * field is packed on `stream` after the work already queued there and copied to dst on the scene's
 * own copy stream, so later substeps on `stream` run while it travels.  dst must stay valid, and
 * should be pinned host memory, until gmpm_read_wait returns.  Two reads may be in flight; a third
 * waits on the device for the oldest. */
gmpm_status gmpm_read_particles_async(gmpm_scene* scene, int field, int dtype, int order, void* dst, size_t bytes,
                                      void* stream);
/* Wait until every overlapped read of the scene has landed. */
gmpm_status gmpm_read_wait(gmpm_scene* scene);

gmpm_status gmpm_read_binning(gmpm_scene* scene, int array, void* dst, size_t bytes);

/* Conservation / CFL diagnostics computed on the device in FP64.  Replaces
 * Particles::getMaxParticleVel_c (Particle_kernal.cu:421-440) used by
 * MPMSimulator::computeDt (Simulator.cpp:200-225). */
gmpm_status gmpm_diagnostics(gmpm_scene* scene, gmpm_diag* out);

const char* gmpm_status_string(gmpm_status status);

/* ---- binning without device allocation -------------------------------------- */

/* Bins caller-owned device positions (interleaved xyz, FP32) by SPGrid page and
 * cell into caller-owned device outputs, allocating no device memory.  It has
 * no counterpart in the reference.  It is for callers that cannot allocate on
 * the call path: a host framework that owns and budgets all device memory and
 * hands this library only views of its own buffers, or a latency-critical loop
 * where cudaMalloc's implicit synchronisation is not allowed.
 *
 * Outputs: perm[i] = input index of sorted slot i and keys_sorted[i] =
 * (page_key << 6) | cell, identical to GMPM_BIN_PERM / GMPM_BIN_KEYS of a scene
 * holding the same positions in the same order (stable sort by key).
 * flags (device pointer, may be NULL) receives the call's GMPM_FLAG_* bits:
 * GMPM_FLAG_OUT_OF_DOMAIN when a position's stencil left the grid (it is then
 * clamped as in the scene binning), GMPM_FLAG_TABLE_OVERFLOW when a cell holds
 * more than 6144 particles (only clamped positions pile up like that); such a
 * cell keeps its scatter order, which can differ from run to run, while every
 * other cell is in canonical order.  The call is asynchronous on `stream`,
 * which must belong to the current device.
 *
 * Limits: n <= GMPM_NOALLOC_MAX_PARTICLES and 8 <= res <= GMPM_NOALLOC_MAX_RES
 * per axis; anything larger returns GMPM_INVALID_ARG before any work.
 * Scratch: one file-scope __device__ array of GMPM_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until process exit.  All calls share
 * it: calls that overlap on the GPU (different streams, or threads without
 * ordering) race and must be serialised by the caller.  The first call on a
 * device resolves the array's address with cudaGetSymbolAddress.  The returned
 * status is that of this call's own API calls and launches. */
#define GMPM_NOALLOC_MAX_PARTICLES 1048576
#define GMPM_NOALLOC_MAX_RES 128
#define GMPM_NOALLOC_SCRATCH_BYTES 21269248
gmpm_status gmpm_bin_positions_noalloc(const float* positions, int64_t n, double dx, int res_x, int res_y, int res_z,
                                       int32_t* perm, uint32_t* keys_sorted, uint32_t* flags, void* stream);

/* ---- synthetic scenes (host only, no device needed) ----------------------- */

/* Seeded synthetic particle sets standing in for the reference's
 * LoadSample::Initial_data / readObj scenes (GPU_MPM/LoadSample.cpp:109-176),
 * whose assets are absent.  Every cell of the body receives `ppc` particles
 * placed uniformly at random inside the cell (splitmix64 stream from `seed`),
 * positions rounded to FP32-representable values so FP32 and FP64 runs start
 * from the same state.
 * Kinds: 0 = notched bar: box of cells[0] x cells[1] x cells[2] cells; the
 *            notch removes the cells with notch_width z-indices centred on
 *            the mid-length of z and y-index < notch_depth (full x extent);
 *        1 = stacked plates: n_plates boxes of cells[] stacked along +y with
 *            gap_cells empty cells between them; material id = plate index;
 *        2 = box (kind 0 without notch).
 * Call with positions == NULL to get the count, then with capacity >= count.
 * material_ids may be NULL. */
typedef struct gmpm_scene_geometry {
    int32_t kind;
    int32_t cells[3];
    int32_t ppc;
    int32_t n_plates;
    int32_t gap_cells;
    int32_t notch_width;
    int32_t notch_depth;
    int32_t _pad0;
    double dx;
    double origin[3];          /* lower corner of the first box */
    uint64_t seed;
} gmpm_scene_geometry;

gmpm_status gmpm_generate_particles(const gmpm_scene_geometry* geom, int64_t* count,
                                    double* positions, int32_t* material_ids, int64_t capacity);

/* ---- the reference's scene samplers (host only) ----------------------------------------------
 * Restatements of the reference's Sample class (GPU_MPM/LoadSample.cpp) that produce the same
 * particles bit for bit.  Each is called first with positions == NULL for the count, then with
 * capacity >= count; positions are xyz-interleaved doubles.  GMPM_IO_ERROR: the file cannot be read. */

/* Sample::readObj (LoadSample.cpp:163-176): one particle per vertex, read as whitespace-separated
 * "<char> x y z" records until a record fails to parse (so an "f a b c" record also yields a
 * particle and a "vn"/"vt" record ends the list, as in the reference), with y shifted by -0.2f. */
gmpm_status gmpm_sample_obj(const char* path, int64_t* count, double* positions, int64_t capacity);

/* Sample::Initialize_Data_cube (LoadSample.cpp:179-213): the cells [N/2 - N/20, N/2 + N/20)^2 x
 * [N/2 - N/8, N/2 + N/8) of an N^3 grid (dx = 1/N), 27 particles per cell on a 3x3x3 lattice of
 * spacing dx/3 around the cell centre. */
gmpm_status gmpm_sample_cube(int32_t n_grid, int64_t* count, double* positions, int64_t capacity);

/* Sample::Initial_data (LoadSample.cpp:109-161): rejection samples of the level set in the SDF file
 * (LoadSDF, :3-32: "ni nj nk", "minx miny minz", "dx", then ni*nj*nk values, i fastest), about 20
 * per grid cell after scaling the level set into the res[] cells around center[] (grid spacing dx).
 * The samples come from the C library's rand() after srand(seed), as the reference draws them from
 * rand() (seed 1 is the generator's initial state, the reference's run): the call reseeds and
 * advances the process-wide generator and is not thread-safe. */
gmpm_status gmpm_sample_sdf(const char* path, const uint32_t center[3], const uint32_t res[3], double dx,
                            uint32_t seed, int64_t* count, double* positions, int64_t capacity);

/* ---- Checkpoint / resume ------------------------------------------------------------------------
 * A binary snapshot of a scene: its description, clock (time, substeps, current dt) and every particle
 * plane of the state in the internal order (the reference's Attribs_Back_Host, Particles.cpp:33-52,
 * and its declared but undefined writePartio, Simulator.h:35, as a restartable file).  Binning and grid
 * are rebuilt by the next substep, so a loaded scene continues bitwise like the original in
 * deterministic mode.  The file is tied to the library's struct layouts (native byte order) and carries
 * a format version: a file written by a build with another particle layout is refused with
 * GMPM_IO_ERROR. */
gmpm_status gmpm_scene_save(gmpm_scene* scene, const char* path);
gmpm_status gmpm_scene_load(gmpm_context* ctx, const char* path, gmpm_scene** out);

/* ---- Batched stepping of independent scenes --------------------------------------------------
 * No reference counterpart: the reference steps one scene per MPMSimulator::simulateStick call
 * (Simulator.cpp:227-259).  A batch advances many independent scenes of uneven size, each with its
 * own grid, with one CUDA graph launch per substep.  Scenes whose kernels are of one kind (precision,
 * P2G mode, energy models, FP64 fallback) advance together with one launch per stage of the substep
 * over a device table of the scenes (23 launches per kind, whatever the number of scenes); scenes
 * with the implicit phase field run their own launch sequences on parallel branches of the graph.
 * Each scene's results are the same as stepping it alone (bitwise in deterministic mode).  The
 * autotuner times candidate launch shapes (the share of SMs each scene's page- and slot-parallel
 * stages are sized for, per scene size class, and the number of concurrent branches) on the first
 * substeps, which are real substeps, and keeps the fastest.
 * Destroy a batch before any of its scenes; a scene may belong to several batches. */
typedef struct gmpm_batch gmpm_batch;

typedef struct gmpm_batch_options {
    int32_t autotune;        /* 1: tune launch shapes on the first substeps (default 1) */
    int32_t trial_substeps;  /* substeps per candidate, even and >= 2 (default 2) */
    int32_t streams;         /* concurrent branches; 0: min(scenes, 32) */
    int32_t sm_share;        /* SMs each scene's launch shapes are sized for when not tuning; 0: all */
} gmpm_batch_options;

typedef struct gmpm_batch_info {
    int32_t n_scenes;
    int32_t streams;          /* concurrent branches in use */
    int32_t tuned;            /* 1 once tuning is finished (or disabled) */
    int32_t n_candidates;     /* launch-shape candidates tried by the tuner */
    int64_t graph_nodes;      /* nodes of one substep graph */
    int64_t captures;         /* graphs captured so far */
    int64_t substeps;         /* batched substeps launched */
    double best_ms_per_substep; /* device time per substep of the chosen candidate (0 if untuned) */
    int32_t sm_share_small;   /* chosen SM share for scenes below 50,000 particles (0: all SMs) */
    int32_t sm_share_medium;  /* ... 50,000 to 200,000 particles */
    int32_t sm_share_large;   /* ... 200,000 particles and above */
    int32_t _pad0;
    double capture_seconds;   /* host time spent capturing and instantiating graphs */
    int64_t kernel_nodes;     /* kernel launches of one substep graph */
    int32_t table_scenes;     /* scenes advanced by one launch per stage (the rest on branches) */
    int32_t _pad1;
} gmpm_batch_info;

void gmpm_batch_options_defaults(gmpm_batch_options* opt);
gmpm_status gmpm_batch_create(gmpm_context* ctx, gmpm_scene* const* scenes, int n_scenes,
                              const gmpm_batch_options* opt /* NULL: defaults */, gmpm_batch** out);
gmpm_status gmpm_batch_substep(gmpm_batch* batch, int n_substeps, void* stream);
gmpm_status gmpm_batch_get_info(gmpm_batch* batch, gmpm_batch_info* out);
gmpm_status gmpm_batch_destroy(gmpm_batch* batch);

/* ---- Serving loop (continuous batching) --------------------------------------------------------
 * No reference counterpart (the reference runs one scene per process from its GLUT loop,
 * gl_main.cpp:304-314).  Requests queue on submit.  Each gmpm_server_step admits queued requests in
 * arrival order while the device-memory budget allows, advances every live scene together through
 * one batch (a CUDA graph launch per substep), never past a request's horizon, and retires requests
 * that reached it: their final position, velocity, F and damage are copied to host memory (FP32,
 * original particle order) and the scene's device memory is freed for waiting requests.  A result
 * does not depend on which requests shared the GPU (bitwise in deterministic mode).  One host
 * thread drives a server. */
typedef struct gmpm_server gmpm_server;

typedef enum gmpm_request_state {
    GMPM_REQUEST_QUEUED = 0,
    GMPM_REQUEST_RUNNING = 1,
    GMPM_REQUEST_DONE = 2,
    GMPM_REQUEST_FAILED = 3
} gmpm_request_state;

typedef struct gmpm_server_options {
    int64_t hbm_budget_bytes;   /* device memory admitted scenes may hold; 0: unlimited (default 120 GB) */
    int32_t max_live;           /* scenes advanced together (default 64; 0: unlimited).  Every change of
                                   the live set re-captures the batch graph, whose size grows with it */
    int32_t autotune;           /* tune the first batch's launch shapes and reuse them (default 1) */
} gmpm_server_options;

typedef struct gmpm_request_status {
    int32_t state;              /* gmpm_request_state */
    int32_t status;             /* gmpm_status of the scene (creation, flags at retirement) */
    int64_t n_particles;
    int64_t substeps_done;
    int64_t horizon;
    double submit_time;         /* seconds since the server was created */
    double admit_time;
    double finish_time;
} gmpm_request_status;

typedef struct gmpm_server_stats {
    int64_t submitted, admitted, completed, failed;
    int64_t live, queued;
    int64_t substeps;           /* batched substeps run */
    int64_t particle_substeps;  /* sum over live scenes of particles x substeps */
    int64_t batches;            /* batches built (one per change of the live set) */
    int64_t device_bytes_in_use;
    int64_t capture_microseconds; /* host time spent capturing batch graphs */
    int64_t admit_microseconds;   /* host time creating admitted scenes */
    int64_t retire_microseconds;  /* host time retiring scenes (waits for their last substeps, reads results) */
    int64_t launch_microseconds;  /* host time enqueueing batched substeps */
} gmpm_server_stats;

void gmpm_server_options_defaults(gmpm_server_options* opt);
gmpm_status gmpm_server_create(gmpm_context* ctx, const gmpm_server_options* opt /* NULL: defaults */,
                               gmpm_server** out);
/* Copies the particle arrays; the scene is created on admission. */
gmpm_status gmpm_server_submit(gmpm_server* srv, const gmpm_scene_desc* desc, const gmpm_particle_init* init,
                               int64_t horizon_substeps, int64_t* request_id);
gmpm_status gmpm_server_step(gmpm_server* srv, int n_substeps, void* stream);
gmpm_status gmpm_server_poll(gmpm_server* srv, int64_t request_id, gmpm_request_status* out);
/* Final field of a finished request: GMPM_FIELD_POSITION, _VELOCITY, _F or _DAMAGE, FP32. */
gmpm_status gmpm_server_read(gmpm_server* srv, int64_t request_id, int field, float* dst, size_t bytes);
/* Forget a finished or failed request (frees its host results). */
gmpm_status gmpm_server_release(gmpm_server* srv, int64_t request_id);
gmpm_status gmpm_server_get_stats(gmpm_server* srv, gmpm_server_stats* out);
gmpm_status gmpm_server_destroy(gmpm_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* GMPM_H */
