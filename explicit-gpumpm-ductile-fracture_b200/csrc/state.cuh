// Device-side views of a scene's particle, binning and grid storage.
//
// Particle state is SoA, one plane per component (stride = capacity), like
// the reference's d_F/d_B planes (Particles.cuh:60-75).  Between substeps the
// state is in the sorted order of the previous binning; the next binning's
// permutation (perm[new] = old, the reference's d_indexTrans) is applied
// while G2P reads it, so no separate reorder pass exists
// (cf. Particles::reorder, Particle_kernal.cu:544-573).
#pragma once
#include <cstdint>

#include "common.cuh"

namespace gmpm {

// Four values of one particle in one aligned word (16 bytes in FP32), so that
// a gather through perm moves them with one wide copy.
template <typename R>
struct __align__(16) Word4 {
    R v[4];
};

// Fields that G2P reads through perm and rewrites in sorted order: double-buffered.
// Only G2P reads F and the plastic state, so those travel as three words per
// particle: fw[0] = (F0, F1, F2, F3), fw[1] = (F4, F5, F6, F7),
// fw[2] = (F8, alpha, psi_max, 0), with F column-major (element (r, c) at
// r + 3c).  The other kernels read x, c and m, which stay one plane each.
template <typename R>
struct PState {
    R* x[3];
    Word4<R>* fw[3];
    R* c;
    R* m;
    uint32_t* id;    // (material << 28) | original index
    int64_t stride;  // elements per plane (>= n + kPlanePad), shared by every particle plane
    __host__ __device__ R& F(int q, int64_t p) const { return fw[q >> 2][p].v[q & 3]; }
    __host__ __device__ R& alpha(int64_t p) const { return fw[2][p].v[1]; }
    __host__ __device__ R& psi(int64_t p) const { return fw[2][p].v[2]; }
};

// Padding of every particle plane beyond n, so a window of kPlanePad previous
// slots can be bulk-copied around any chunk without leaving the allocation.
constexpr int kPlanePad = 1024;

// Fields that only G2P writes and only the next P2G reads: single-buffered.
template <typename R>
struct PAux {
    R* v[3];
    R* B[9];
    R* sigma[6];  // V0 P F^T: xx yy zz xy xz yz
    R* vol;       // V0 det F
    R* FP;
    R* q[3];      // 4 L0^2 V grad c
};

struct BinDev {
    uint32_t* keys;         // [n] (page_key << 6) | cell, previous order
    uint32_t* keys_sorted;  // [n] sorted keys
    int32_t* perm;          // [n] new slot -> previous slot
    uint8_t* page_flag;     // [key_space]
    int32_t* page_rank;     // [key_space] exclusive scan of page_flag
    uint8_t* grid_flag;     // [key_space]
    int32_t* grid_rank;     // [key_space]
    uint32_t* block_keys;   // [nb_cap]
    int32_t* cell_count;    // [nb_cap*64] histogram, then scatter fill counters
    int32_t* cell_start;    // [nb_cap*64 + 1]
    uint32_t* grid_keys;    // [ng_cap]
    int32_t* adj;           // [nb_cap*8]  grid index of page + (i,j,k), slot 4i+2j+k
    int32_t* grid_src;      // [ng_cap*8]  particle page of grid page - (i,j,k), or -1
    int32_t nb_cap;
    int32_t ng_cap;
    uint32_t key_space;
    int64_t n;
};

}  // namespace gmpm
