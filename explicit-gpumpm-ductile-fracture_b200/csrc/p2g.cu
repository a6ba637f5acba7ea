// P2G: APIC particle-to-grid transfer on SPGrid pages (P2G_APIC,
// P2GKernal.cu:512-702) plus the phase-field channels (volP2G_APIC,
// preConditionP2G_APIC, AxP2G_APIC: P2GKernal.cu:897-1326).
//
// One CTA per particle page.  A page's particles share the page's 6x6x6 node
// window and, within a cell, the same 3x3x3 stencil.  Thread (cell, i, j)
// owns the three stencil nodes (i, j, 0..2) of its cell and loops over the
// cell's particles in sorted order, accumulating 9 channels x 3 nodes in
// registers — no shuffles, no atomics.  The per-(cell,i,j) partials are then
// gathered per window node in fixed cell order and written once to the page's
// tile in HBM; the grid kernel sums the eight tiles overlapping each grid page
// in fixed slot order.  The result is bitwise reproducible run to run.
#include <cstdint>

#include "kernels.h"

namespace gmpm {

constexpr int kP2GThreads = 576;  // 64 cells x 9 stencil columns

template <typename R> struct P2GChunk;
template <> struct P2GChunk<float> { static constexpr int value = 256; };
template <> struct P2GChunk<double> { static constexpr int value = 128; };

// Staged per-particle quantities (SoA in shared memory).
enum StageField : int {
    SF_WX = 0, SF_GX = 3, SF_WY = 6, SF_GY = 9, SF_WZ = 12, SF_GZ = 15,
    SF_M = 18, SF_C = 19, SF_V = 20, SF_VFP = 21,
    SF_U = 22,    // m v - m B D^-1 xp            (3)
    SF_A = 25,    // dx m B D^-1, (r,c) at 3r+c   (9)
    SF_S = 34,    // -dt V0 P F^T: xx yy zz xy xz yz (6)
    SF_Q = 40,    // 4 L0^2 V grad c              (3)
    kStage = 43
};

template <typename R>
__device__ __forceinline__ void bspline1d(R xp, R inv_dx, R* w, R* g) {
    // quadratic B-spline weights and gradients on nodes base+0..2, xp relative
    // to the base node (P2GKernal.cu:590-611)
    R d0 = xp * inv_dx;
    R z = R(1.5) - d0;
    w[0] = R(0.5) * z * z;
    g[0] = -z * inv_dx;
    d0 = d0 - R(1);
    w[1] = R(0.75) - d0 * d0;
    g[1] = -d0 * R(2) * inv_dx;
    z = R(1.5) - (R(1) - d0);
    w[2] = R(0.5) * z * z;
    g[2] = z * inv_dx;
}

template <typename R>
__global__ void __launch_bounds__(kP2GThreads, 1)
    k_p2g(const SceneDev<R>* __restrict__ sc, PState<R> st, PAux<R> aux, BinDev bin, R* __restrict__ tile,
          const Counters* __restrict__ cnt) {
    constexpr int CH = P2GChunk<R>::value;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* stage = reinterpret_cast<R*>(smem_raw);
    R* partial = stage + kStage * CH;

    const int t = threadIdx.x;
    const int my_cell = t / 9;
    const int ij = t - my_cell * 9;
    const int my_i = ij / 3, my_j = ij - (ij / 3) * 3;
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const R dx = sc->dx, inv_dx = sc->inv_dx, dt = sc->dt, Dinv = sc->Dinv;
    const R fi = R(my_i), fj = R(my_j);

    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        const int32_t* cs = bin.cell_start + (int64_t)b * 64;
        const int bs = cs[0], be = cs[64];
        const int my_lo = cs[my_cell], my_hi = cs[my_cell + 1];
        int bx, by, bz;
        page_coords(bin.block_keys[b], bx, by, bz);

        R acc[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) acc[q] = R(0);

        for (int c0 = bs; c0 < be; c0 += CH) {
            const int cn = min(CH, be - c0);
            // ---- stage the chunk's particles (gathered through perm) ----
            for (int p = t; p < cn; p += kP2GThreads) {
                const int slot = c0 + p;
                const int o = bin.perm[slot];
                const uint32_t cell = bin.keys_sorted[slot] & 63u;
                const int base[3] = {4 * bx + (int)(cell >> 4), 4 * by + (int)((cell >> 2) & 3), 4 * bz + (int)(cell & 3)};
                R xp[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) xp[a] = st.x[a][o] - R(base[a]) * dx;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    R w[3], g[3];
                    bspline1d(xp[a], inv_dx, w, g);
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        stage[(SF_WX + 6 * a + q) * CH + p] = w[q];
                        stage[(SF_GX + 6 * a + q) * CH + p] = g[q];
                    }
                }
                const R m = st.m[o];
                const R V = aux.vol[o];
                stage[SF_M * CH + p] = m;
                stage[SF_C * CH + p] = st.c[o];
                stage[SF_V * CH + p] = V;
                stage[SF_VFP * CH + p] = V * aux.FP[o];
                R mB[9];  // m B D^-1, (r,c) at 3r+c; stored column-major (r + 3c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) mB[3 * r + c] = m * aux.B[r + 3 * c][o] * Dinv;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const R u = m * aux.v[r][o] - (mB[3 * r] * xp[0] + mB[3 * r + 1] * xp[1] + mB[3 * r + 2] * xp[2]);
                    stage[(SF_U + r) * CH + p] = u;
#pragma unroll
                    for (int c = 0; c < 3; ++c) stage[(SF_A + 3 * r + c) * CH + p] = dx * mB[3 * r + c];
                }
#pragma unroll
                for (int q = 0; q < 6; ++q) stage[(SF_S + q) * CH + p] = -dt * aux.sigma[q][o];
#pragma unroll
                for (int a = 0; a < 3; ++a) stage[(SF_Q + a) * CH + p] = aux.q[a][o];
            }
            __syncthreads();
            // ---- accumulate this thread's stencil column over its cell ----
            const int lo = max(my_lo, c0), hi = min(my_hi, c0 + cn);
            for (int s = lo; s < hi; ++s) {
                const int p = s - c0;
                const R wx = stage[(SF_WX + my_i) * CH + p], gx = stage[(SF_GX + my_i) * CH + p];
                const R wy = stage[(SF_WY + my_j) * CH + p], gy = stage[(SF_GY + my_j) * CH + p];
                const R wxy = wx * wy, gxy0 = gx * wy, gxy1 = wx * gy;
                const R mW = stage[SF_M * CH + p] * wxy;
                const R cW = stage[SF_C * CH + p] * wxy;
                const R VW = stage[SF_V * CH + p] * wxy;
                const R FW = stage[SF_VFP * CH + p] * wxy;
                const R Sxx = stage[(SF_S + 0) * CH + p], Syy = stage[(SF_S + 1) * CH + p];
                const R Szz = stage[(SF_S + 2) * CH + p], Sxy = stage[(SF_S + 3) * CH + p];
                const R Sxz = stage[(SF_S + 4) * CH + p], Syz = stage[(SF_S + 5) * CH + p];
                // force terms: dt f_r = (S_r0 gxy0 + S_r1 gxy1) wz + S_r2 wxy gz
                const R al0 = Sxx * gxy0 + Sxy * gxy1, be0 = Sxz * wxy;
                const R al1 = Sxy * gxy0 + Syy * gxy1, be1 = Syz * wxy;
                const R al2 = Sxz * gxy0 + Syz * gxy1, be2 = Szz * wxy;
                const R gam = stage[(SF_Q + 0) * CH + p] * gxy0 + stage[(SF_Q + 1) * CH + p] * gxy1;
                const R del = stage[(SF_Q + 2) * CH + p] * wxy;
                R u0 = stage[(SF_U + 0) * CH + p] + stage[(SF_A + 0) * CH + p] * fi + stage[(SF_A + 1) * CH + p] * fj;
                R u1 = stage[(SF_U + 1) * CH + p] + stage[(SF_A + 3) * CH + p] * fi + stage[(SF_A + 4) * CH + p] * fj;
                R u2 = stage[(SF_U + 2) * CH + p] + stage[(SF_A + 6) * CH + p] * fi + stage[(SF_A + 7) * CH + p] * fj;
                const R a02 = stage[(SF_A + 2) * CH + p], a12 = stage[(SF_A + 5) * CH + p],
                        a22 = stage[(SF_A + 8) * CH + p];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const R wz = stage[(SF_WZ + k) * CH + p], gz = stage[(SF_GZ + k) * CH + p];
                    const R w = wxy * wz;
                    R* A = acc + 9 * k;
                    A[CH_M] += mW * wz;
                    A[CH_P0] += w * u0 + al0 * wz + be0 * gz;
                    A[CH_P1] += w * u1 + al1 * wz + be1 * gz;
                    A[CH_P2] += w * u2 + al2 * wz + be2 * gz;
                    A[CH_CW] += cW * wz;
                    A[CH_W] += w;
                    A[CH_VW] += VW * wz;
                    A[CH_VWFP] += FW * wz;
                    A[CH_KC] += gam * wz + del * gz;
                    u0 += a02;
                    u1 += a12;
                    u2 += a22;
                }
            }
            __syncthreads();
        }
        // ---- fixed-order gather of the partials into the page tile ----
#pragma unroll
        for (int q = 0; q < 27; ++q) partial[t * 27 + q] = acc[q];
        __syncthreads();
        R* out = tile + (int64_t)b * kP2GChannels * kWindowNodes;
        for (int oi = t; oi < kP2GChannels * kWindowNodes; oi += kP2GThreads) {
            const int ch = oi / kWindowNodes;
            const int node = oi - ch * kWindowNodes;
            const int a = node / 36, bb = (node / 6) % 6, cc = node % 6;
            R sum = R(0);
            for (int cx = max(0, a - 2); cx <= min(3, a); ++cx)
                for (int cy = max(0, bb - 2); cy <= min(3, bb); ++cy)
                    for (int cz = max(0, cc - 2); cz <= min(3, cc); ++cz) {
                        const int cell = cx * 16 + cy * 4 + cz;
                        const int col = cell * 9 + (a - cx) * 3 + (bb - cy);
                        sum += partial[col * 27 + (cc - cz) * 9 + ch];
                    }
            out[oi] = sum;
        }
        __syncthreads();
    }
}

template <typename R>
size_t p2g_smem_bytes() {
    return sizeof(R) * ((size_t)kStage * P2GChunk<R>::value + (size_t)kP2GThreads * 27);
}

template <typename R>
cudaError_t launch_p2g(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const size_t smem = p2g_smem_bytes<R>();
    k_p2g<R><<<cfg.num_sms, kP2GThreads, smem, stream>>>(sc, st, aux, bin, reinterpret_cast<R*>(grid.tile), cnt);
    return cudaGetLastError();
}

template <typename R>
cudaError_t prepare_p2g() {
    return cudaFuncSetAttribute(k_p2g<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_smem_bytes<R>());
}
template cudaError_t prepare_p2g<float>();
template cudaError_t prepare_p2g<double>();

template cudaError_t launch_p2g<float>(const SceneDev<float>*, const PState<float>&, const PAux<float>&, BinDev,
                                       GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_p2g<double>(const SceneDev<double>*, const PState<double>&, const PAux<double>&, BinDev,
                                        GridDev, Counters*, LaunchCfg, cudaStream_t);

}  // namespace gmpm
