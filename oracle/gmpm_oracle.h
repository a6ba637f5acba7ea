/*
 * ORACLE — test infrastructure only, never the product.
 *
 * FP64 CPU restatement of the reference's explicit APIC-MPM substep
 * (KemengHuang/Explicit-GPUMPM-Ductile-Fracture, GPU_MPM/).  The reference has
 * no CPU path; this file restates its kernels so tests can check the CUDA
 * library against it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it.
 *
 * Pinning: the SPGrid masks and Linear_Offset, the material constants and the
 * 3x3 SVD are checked against the reference's own code compiled here
 * (oracle/_ref/ref_kat), and so are the per-thread kernels applyVonMises,
 * computePhase_field_vol, undateGrid_kernal, collideWithGround, PullGrid_kernal,
 * cal_cellId and calcIndex, run serially on the host (oracle/_ref/ref_kernels);
 * fixtures in tests/golden/.  P2G_APIC, G2P_APIC and the binning use shared
 * memory, warp reductions and atomics; they are checked by invariants and
 * hand-derived identities.
 */
#ifndef GMPM_ORACLE_H
#define GMPM_ORACLE_H

#include <stdint.h>
#include "gmpm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SPGrid bit arithmetic. */
void     orc_masks(uint64_t out[3]);
uint64_t orc_bit_spread(uint64_t mask, int64_t data);
uint64_t orc_linear_offset(int i, int j, int k);
uint64_t orc_packed_add(uint64_t a, uint64_t b);
int64_t  orc_bit_pack(uint64_t mask, uint64_t data);

/* 3x3 SVD: F row-major in, U/V row-major and S out (F = U diag(S) V^T). */
void orc_svd3(const double* F_rowmajor, double* U_rowmajor, double* S, double* V_rowmajor);

/* Material constants lambda, mu, kappa (Materials.cpp:4-13). */
void orc_lame(double E, double nu, double* lambda, double* mu, double* kappa);

/* One applyVonMises update of a single particle.
 * io[0..8] F col-major, io[9] g, io[10] alpha, io[11] c, io[12] psi_max.
 * out: [0..8] F, [9] g_new, [10] alpha, [11] psi_max, [12] FP,
 *      [13..21] contribution V0*P*F^T col-major, [22] V0*det F. */
void orc_von_mises(const gmpm_material* mat, double V0, const double* io, double* out);

/* The same update through the material's energy model (mat->energy_model:
 * von Mises, fixed-corotated or Neo-Hookean with fracture); dx sets the
 * Neo-Hookean phase-field length L0 = dx/2.  Same io / out layout. */
void orc_constitutive(const gmpm_material* mat, double V0, double dx, const double* io, double* out);

/* Stencil base node floor(x/dx + 0.5) - 1 of one particle (cal_cellId,
 * Particle_kernal.cu:158-165, and calcIndex, TimeIntegrator.cu:53-61), clamped
 * into [0, res - 3] per axis; returns GMPM_FLAG_OUT_OF_DOMAIN if it was not
 * inside. */
int orc_base_node(double inv_dx, const int32_t res[3], const double x[3], int32_t out[3]);

/* One grid node of the grid update (undateGrid_kernal, TimeIntegrator.cu:63-111)
 * followed by the scene's velocity conditions (slabs, spheres as in
 * PullGrid_kernal :169-214, sticky walls as in collideWithGround :117-165) at
 * simulated time t.  ch: mass, momentum xyz, force xyz, sum w c, sum w.
 * out: velocity xyz, c = sum w c / sum w (FP64 division). */
void orc_grid_node(const gmpm_scene_desc* desc, double t, const int32_t node[3], const double ch[9], double out[4]);

/* Scene set-up without the product library (the CPU legs of the benchmark):
 * the reference-default description and the seeded synthetic particles, equal
 * field for field and bit for bit to gmpm_scene_desc_reference_defaults and
 * gmpm_generate_particles. */
int orc_scene_desc_reference_defaults(gmpm_scene_desc* d, double dx, int rx, int ry, int rz);
int orc_generate_particles(const gmpm_scene_geometry* g, int64_t* count, double* positions, int32_t* material_ids,
                           int64_t capacity);

typedef struct orc_scene orc_scene;

orc_scene* orc_scene_create(const gmpm_scene_desc* desc, int64_t n, const double* pos,
                            const double* vel, const double* mass, const int32_t* mat_ids);
void orc_scene_destroy(orc_scene* s);
void orc_set_threads(int n);
int  orc_get_threads(void);

/* Run n substeps; returns accumulated GMPM_FLAG_* bits. */
uint32_t orc_substep(orc_scene* s, int n);
/* Binning only (canonical stable sort by (key, previous slot)). */
uint32_t orc_rebin(orc_scene* s);

int64_t orc_num_particles(const orc_scene* s);
int64_t orc_num_blocks(const orc_scene* s);
int64_t orc_num_grid_blocks(const orc_scene* s);

/* Field copy in the oracle's current (sorted) order; layout as gmpm_field. */
void orc_get_field(const orc_scene* s, int field, double* out);
/* Binning array copy; layout and types as gmpm_binning_array. */
void orc_get_binning(const orc_scene* s, int array, void* out);
void orc_diagnostics(const orc_scene* s, gmpm_diag* out);

#ifdef __cplusplus
}
#endif
#endif
