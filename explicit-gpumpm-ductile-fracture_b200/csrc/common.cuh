// Shared device definitions: scene parameters as the kernels see them, SPGrid
// page keys, status flags.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gmpm.h"

namespace gmpm {

constexpr int kMaxMaterials = GMPM_MAX_MATERIALS;
constexpr int kCellsPerBlock = 64;   // 4x4x4 nodes per SPGrid page (SPGridMask.cpp:76-89)
constexpr int kWindow = 6;           // a page's particles touch a 6x6x6 node window
constexpr int kWindowNodes = 216;

// P2G channels written to the per-page tile scratch.  Momentum already
// includes dt * force (the reference adds f*dt/m after dividing p by m,
// TimeIntegrator.cu:96-107; both are sums over the same particles).
enum P2GChannel : int {
    CH_M = 0,      // sum m w
    CH_P0 = 1,     // sum m w (v + B D^-1 (x_i - x_p)) - dt V0 P F^T grad w
    CH_P1 = 2,
    CH_P2 = 3,
    CH_CW = 4,     // sum w c
    CH_W = 5,      // sum w
    CH_VW = 6,     // sum V w
    CH_VWFP = 7,   // sum V w FP
    CH_KC = 8,     // sum grad w . (4 L0^2 V grad c)
    kP2GChannels = 9
};

// Grid channels read by G2P.
enum GridChannel : int { GC_V0 = 0, GC_V1 = 1, GC_V2 = 2, GC_DC = 3, GC_CN = 4, kGridChannels = 5 };

// Per-material constants in the precision of the kernel.
template <typename Real>
struct MaterialDev {
    Real lambda, mu, kappa;
    Real D[9];              // inverse of the isotropic stiffness (Gauss-Jordan as in Inverse())
    Real yield_stress, hardening;
    int hardening_law;
    int energy_model;       // gmpm_energy_model
    Real alpha_cap, dlambda_cap, strain_cap, psi_cap;
    Real fracture_energy, softening_onset, residual_fracture;
    Real theta, length_scale, mobility;
    Real one_minus_theta;   // (1 - theta) rounded to float: theta is a float in the reference (:334)
};

// Velocity conditions: axis-aligned slabs and moving spheres.  Kept as one
// contiguous block so the host can replace it with a single copy.
template <typename Real>
struct VelocityConditions {
    int n_slabs, n_spheres;
    int slab_axis[GMPM_MAX_SLAB_BCS];
    Real slab_lo[GMPM_MAX_SLAB_BCS], slab_hi[GMPM_MAX_SLAB_BCS], slab_vel[GMPM_MAX_SLAB_BCS][3];
    Real sph_c[GMPM_MAX_SPHERE_BCS][3], sph_r[GMPM_MAX_SPHERE_BCS], sph_v[GMPM_MAX_SPHERE_BCS][3];
};

template <typename Real>
struct SceneDev {
    Real dx, inv_dx, dt;
    Real Dinv;              // 4 / dx^2 (Setting.h:17)
    Real gravity[3];
    Real V0;
    int res[3];
    int key_bits;           // bits per axis of the page key space
    int n_materials;
    MaterialDev<Real> mat[kMaxMaterials];
    int wall_bc, wall_layers;
    VelocityConditions<Real> bc;
    int phase_field;
    int fp64_svd_fallback;  // precision mode 2
    Real svd_fallback_ratio;
    Real mobility;          // scene mobility used by the grid phase-field update (material 0)
    double dx_d, inv_dx_d;  // binning arithmetic is always FP64
    int adaptive_dt;        // CFL time step from the previous G2P's max speed
    int pcg_max_combine;    // implicit phase field: combine partial dot products by max (reference quirk)
    double pcg_tolerance;   // implicit phase field: stop when max |r| < tolerance
    double dt_max;          // the scene's dt: upper bound of the adaptive step
    double cfl_dx;          // cfl_number * dx
};

// Counters and flags living in device memory (written by kernels, read by host on demand).
struct Counters {
    int n_blocks;
    int n_grid_blocks;
    unsigned int flags;
    int pad;
    double time;
    long long substeps;
    unsigned long long vmax2_bits;  // max |v_p|^2 of the last G2P (FP64 bits; non-negative, so integer order)
    int pcg_iterations;             // implicit phase field: iterations of the last solve
    int pad2;
};

// Compensated (Kahan) summation: s += v with the low-order error carried in c.
template <typename R>
__device__ __forceinline__ void kahan_add(R& s, R& c, R v) {
    const R y = v - c;
    const R t = s + y;
    c = (t - s) - y;
    s = t;
}

// ---- SPGrid page keys -----------------------------------------------------
// The page key of block (bx,by,bz) is offset>>12 of SPGridMask::Linear_Offset:
// Morton interleave with z in bit 0, y in bit 1, x in bit 2 (SPGridMask.cpp:97-105).
__host__ __device__ inline uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__host__ __device__ inline uint32_t compact3(uint32_t v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030c30c3u;
    v = (v | (v >> 4)) & 0x0300f00fu;
    v = (v | (v >> 8)) & 0x030000ffu;
    v = (v | (v >> 16)) & 0x000003ffu;
    return v;
}
__host__ __device__ inline uint32_t page_key(int bx, int by, int bz) {
    return spread3((uint32_t)bz) | (spread3((uint32_t)by) << 1) | (spread3((uint32_t)bx) << 2);
}
__host__ __device__ inline void page_coords(uint32_t key, int& bx, int& by, int& bz) {
    bz = (int)compact3(key);
    by = (int)compact3(key >> 1);
    bx = (int)compact3(key >> 2);
}

__device__ inline void raise_flag(Counters* c, unsigned int f) { atomicOr(&c->flags, f); }

// Cell key of a position, (page_key << 6) | cell of the base node, with the
// base node (int)(x / dx + 0.5) - 1 in FP64 as in cal_cellId
// (Particle_kernal.cu:162-164).  A base node whose 3-node stencil would leave
// the grid is clamped to its edge and sets `bad`.  Shared by the binning's key
// pass and G2P, which keys the positions it writes.
template <typename R>
__device__ __forceinline__ uint32_t cell_key(const R x[3], double inv_dx, const int res[3], bool& bad) {
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int hi = res[a] - 3;
        const double t = __dadd_rn(__dmul_rn((double)x[a], inv_dx), 0.5);
        if (!(t >= 1.0)) {
            base[a] = 0;
            bad = true;
        } else if (t >= (double)(hi + 2)) {
            base[a] = hi;
            bad = true;
        } else {
            base[a] = (int)t - 1;
        }
    }
    const uint32_t cell = (uint32_t)(((base[0] & 3) << 4) | ((base[1] & 3) << 2) | (base[2] & 3));
    return (page_key(base[0] >> 2, base[1] >> 2, base[2] >> 2) << 6) | cell;
}

// ---- launches over one scene or many ------------------------------------------
// A kernel body sees its CTA's index and the CTA count of its scene's share of
// the launch: the CUDA block index and grid size in a one-scene launch, or the
// CTA's place in its scene's range in a batched launch over many scenes.
struct VB {
    int b, g;
};
__device__ __forceinline__ VB own_blocks() { return VB{(int)blockIdx.x, (int)gridDim.x}; }

// Batched launch: scene s owns CTAs [start[s], start[s + 1]) (n_scenes + 1
// entries, every scene at least one CTA).  Returns the scene of this CTA and
// its place in the scene's range.
__device__ __forceinline__ int scene_of_block(const int32_t* __restrict__ start, int n_scenes, VB& v) {
    const int b = (int)blockIdx.x;
    int lo = 0, hi = n_scenes - 1;  // the last scene whose range starts at or before b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&start[mid]) <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int s0 = __ldg(&start[lo]);
    v.b = b - s0;
    v.g = __ldg(&start[lo + 1]) - s0;
    return lo;
}

}  // namespace gmpm
