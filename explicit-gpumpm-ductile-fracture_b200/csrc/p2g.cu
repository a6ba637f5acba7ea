// P2G: APIC particle-to-grid transfer on SPGrid pages (P2G_APIC,
// P2GKernal.cu:512-702) plus the phase-field channels (volP2G_APIC,
// preConditionP2G_APIC, AxP2G_APIC: P2GKernal.cu:897-1326).
//
// One CTA per particle page (grid-stride).  A page's particles share the
// page's 6x6x6 node window and, within a cell, the same 3x3x3 stencil.  The
// page's particles (sorted by cell) are staged at once (in chunks only for
// pages above 512 particles), gathered through perm into one 36-word record
// each in shared memory: x/y offsets, z weights, mass, damage, APIC affine
// terms, stress and phase-field flux.
//
// Work split: 16 cell z-columns (cx, cy) x 9 stencil columns (i, j) x 2
// channel groups.  Thread (cx, cy, i, j, group) sweeps the cells
// (cx, cy, 0..3) in order and owns window nodes (cx+i, cy+j, 0..5) for its
// group's channels: group 0 = momentum x, y + mass + damage weight, group 1 =
// momentum z + weight + the three phase-field channels.  Every particle of
// cell cz adds to nodes cz..cz+2 with register indices fixed at compile time
// (the sweep over cz is unrolled), so the sums stay in registers: no
// shuffles and no per-particle atomics.
//
// Deterministic mode: the column sums are gathered per window node in a fixed
// order (at most 9 terms) and written once to the page's tile in HBM, so
// results are bitwise reproducible.  Fast mode: columns add into a shared
// tile with atomics.  The grid kernel sums the eight page tiles overlapping
// each grid page in fixed slot order either way.
#include <cstdint>

#include "kernels.h"

namespace gmpm {

constexpr int kColumns = 144;       // 16 cell z-columns x 9 stencil columns
constexpr int kGroupThreads = 160;  // 5 warps per channel group (144 busy)
constexpr int kP2GThreads = 2 * kGroupThreads;
constexpr int kRec = 36;            // words per staged particle record
constexpr int kColAcc = 54;         // 6 z-nodes x 9 channels

template <typename R> struct P2GChunk;
template <> struct P2GChunk<float> { static constexpr int value = 512; };
template <> struct P2GChunk<double> { static constexpr int value = 256; };

// Staged record layout (words); groups of four are read as 16-byte words.
enum RecField : int {
    RF_XP0 = 0, RF_XP1 = 1, RF_M = 2, RF_C = 3,
    RF_WZ = 4,                  // wz0 wz1 wz2
    RF_GZ = 7,                  // gz0 gz1 gz2
    RF_U = 10,                  // m v - m B D^-1 xp          (3)
    RF_A = 13,                  // dx m B D^-1, (r,c) at 3r+c (9)
    RF_SXX = 22, RF_SYY = 23, RF_SZZ = 24, RF_SXY = 25, RF_SXZ = 26, RF_SYZ = 27,  // -dt V0 P F^T
    RF_V = 28, RF_VFP = 29,
    RF_Q = 30,                  // 4 L0^2 V grad c            (3)
    RF_PAD = 33
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
__device__ __forceinline__ void stage_particle(const SceneDev<R>* __restrict__ sc, const PState<R>& st,
                                              const PAux<R>& aux, int o, const int base[3], R* rec) {
    const R dx = sc->dx, inv_dx = sc->inv_dx, dt = sc->dt, Dinv = sc->Dinv;
    R xp[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xp[a] = st.x[a][o] - R(base[a]) * dx;
    rec[RF_XP0] = xp[0];
    rec[RF_XP1] = xp[1];
    {
        R w[3], g[3];
        bspline1d(xp[2], inv_dx, w, g);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            rec[RF_WZ + q] = w[q];
            rec[RF_GZ + q] = g[q];
        }
    }
    const R m = st.m[o];
    const R V = aux.vol[o];
    rec[RF_M] = m;
    rec[RF_C] = st.c[o];
    rec[RF_V] = V;
    rec[RF_VFP] = V * aux.FP[o];
    R mB[9];  // m B D^-1, (r,c) at 3r+c; B planes are column-major (r + 3c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) mB[3 * r + c] = m * aux.B[r + 3 * c][o] * Dinv;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        rec[RF_U + r] = m * aux.v[r][o] - (mB[3 * r] * xp[0] + mB[3 * r + 1] * xp[1] + mB[3 * r + 2] * xp[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) rec[RF_A + 3 * r + c] = dx * mB[3 * r + c];
    }
    rec[RF_SXX] = -dt * aux.sigma[0][o];
    rec[RF_SYY] = -dt * aux.sigma[1][o];
    rec[RF_SZZ] = -dt * aux.sigma[2][o];
    rec[RF_SXY] = -dt * aux.sigma[3][o];
    rec[RF_SXZ] = -dt * aux.sigma[4][o];
    rec[RF_SYZ] = -dt * aux.sigma[5][o];
#pragma unroll
    for (int a = 0; a < 3; ++a) rec[RF_Q + a] = aux.q[a][o];
    rec[RF_PAD] = rec[RF_PAD + 1] = rec[RF_PAD + 2] = R(0);
}

// Per-thread constants of the B-spline piece of stencil node i along one
// axis, written around z = xp/dx - shift: w = a z^2 + b, dw/dx = c z.
template <typename R>
struct Piece {
    R shift, a, b, c;
    __device__ __forceinline__ void init(int i, R inv_dx) {
        shift = i == 0 ? R(1.5) : (i == 1 ? R(1) : R(0.5));
        a = i == 1 ? R(-1) : R(0.5);
        b = i == 1 ? R(0.75) : R(0);
        c = (i == 1 ? R(-2) : R(1)) * inv_dx;
    }
    __device__ __forceinline__ void eval(R xp_over_dx, R& w, R& g) const {
        const R z = xp_over_dx - shift;
        w = a * (z * z) + b;
        g = c * z;
    }
};

template <typename R>
__device__ __forceinline__ void load_record(const R* __restrict__ rec_s, R* rec) {
    static_assert((kRec * sizeof(R)) % 16 == 0, "record must be whole 16-byte words");
#pragma unroll
    for (int q = 0; q < (int)(kRec * sizeof(R) / 16); ++q)
        reinterpret_cast<uint4*>(rec)[q] = reinterpret_cast<const uint4*>(rec_s)[q];
}

// Group 0: momentum x, y (incl. dt force), mass, damage weight.
// acc: 6 z-nodes x {M, P0, P1, CW}.
template <int CZ, typename R>
__device__ __forceinline__ void accumulate_g0(const R* __restrict__ rec_s, const Piece<R>& px, const Piece<R>& py,
                                              R inv_dx, R fi, R fj, R* acc) {
    R rec[kRec];
    load_record(rec_s, rec);
    R wx, gx, wy, gy;
    px.eval(rec[RF_XP0] * inv_dx, wx, gx);
    py.eval(rec[RF_XP1] * inv_dx, wy, gy);
    const R wxy = wx * wy, gxy0 = gx * wy, gxy1 = wx * gy;
    const R mW = rec[RF_M] * wxy, cW = rec[RF_C] * wxy;
    // dt f_r = (S_r0 gxy0 + S_r1 gxy1) wz + S_r2 wxy gz
    const R al0 = rec[RF_SXX] * gxy0 + rec[RF_SXY] * gxy1, be0 = rec[RF_SXZ] * wxy;
    const R al1 = rec[RF_SXY] * gxy0 + rec[RF_SYY] * gxy1, be1 = rec[RF_SYZ] * wxy;
    R u0 = rec[RF_U + 0] + rec[RF_A + 0] * fi + rec[RF_A + 1] * fj;
    R u1 = rec[RF_U + 1] + rec[RF_A + 3] * fi + rec[RF_A + 4] * fj;
    const R a02 = rec[RF_A + 2], a12 = rec[RF_A + 5];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R wz = rec[RF_WZ + k], gz = rec[RF_GZ + k];
        const R w = wxy * wz;
        R* A = acc + 4 * (CZ + k);
        A[0] += mW * wz;
        A[1] += w * u0 + al0 * wz + be0 * gz;
        A[2] += w * u1 + al1 * wz + be1 * gz;
        A[3] += cW * wz;
        u0 += a02;
        u1 += a12;
    }
}

// Group 1: momentum z (incl. dt force), weight, V w, V w FP, grad w . q.
// acc: 6 z-nodes x {P2, W, VW, VWFP, KC}.
template <int CZ, typename R>
__device__ __forceinline__ void accumulate_g1(const R* __restrict__ rec_s, const Piece<R>& px, const Piece<R>& py,
                                              R inv_dx, R fi, R fj, R* acc) {
    R rec[kRec];
    load_record(rec_s, rec);
    R wx, gx, wy, gy;
    px.eval(rec[RF_XP0] * inv_dx, wx, gx);
    py.eval(rec[RF_XP1] * inv_dx, wy, gy);
    const R wxy = wx * wy, gxy0 = gx * wy, gxy1 = wx * gy;
    const R VW = rec[RF_V] * wxy, FW = rec[RF_VFP] * wxy;
    const R al2 = rec[RF_SXZ] * gxy0 + rec[RF_SYZ] * gxy1, be2 = rec[RF_SZZ] * wxy;
    const R gam = rec[RF_Q + 0] * gxy0 + rec[RF_Q + 1] * gxy1, del = rec[RF_Q + 2] * wxy;
    R u2 = rec[RF_U + 2] + rec[RF_A + 6] * fi + rec[RF_A + 7] * fj;
    const R a22 = rec[RF_A + 8];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R wz = rec[RF_WZ + k], gz = rec[RF_GZ + k];
        const R w = wxy * wz;
        R* A = acc + 5 * (CZ + k);
        A[0] += w * u2 + al2 * wz + be2 * gz;
        A[1] += w;
        A[2] += VW * wz;
        A[3] += FW * wz;
        A[4] += gam * wz + del * gz;
        u2 += a22;
    }
}

template <int G, int CZ, typename R>
__device__ __forceinline__ void sweep_cell(const R* __restrict__ stage, const int* __restrict__ s_cs, int cb, int c0,
                                           int c1, const Piece<R>& px, const Piece<R>& py, R inv_dx, R fi, R fj,
                                           R* acc) {
    const int lo = max(s_cs[cb + CZ], c0) - c0, hi = min(s_cs[cb + CZ + 1], c1) - c0;
    for (int p = lo; p < hi; ++p) {
        if (G == 0)
            accumulate_g0<CZ>(stage + (size_t)p * kRec, px, py, inv_dx, fi, fj, acc);
        else
            accumulate_g1<CZ>(stage + (size_t)p * kRec, px, py, inv_dx, fi, fj, acc);
    }
}

// Channel (CH_*) of slot Q of group G's accumulator row.
template <int G, int Q>
struct GroupChannel {
    static constexpr int value = G == 0 ? (Q == 0 ? CH_M : Q == 1 ? CH_P0 : Q == 2 ? CH_P1 : CH_CW)
                                        : (Q == 0 ? CH_P2 : Q == 1 ? CH_W : Q == 2 ? CH_VW : Q == 3 ? CH_VWFP : CH_KC);
};

template <int G, int Q, typename R, bool kDeterministic>
__device__ __forceinline__ void flush_channel(const R* acc, R* acc_smem, int l, int a, int bb) {
    constexpr int NG = G == 0 ? 4 : 5;
    constexpr int ch = GroupChannel<G, Q>::value;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        if (kDeterministic)
            acc_smem[(size_t)l * kColAcc + c * 9 + ch] = acc[c * NG + Q];
        else
            atomicAdd(&acc_smem[ch * kWindowNodes + a * 36 + bb * 6 + c], acc[c * NG + Q]);
    }
}

// Sweep the z-column over the chunk [c0, c1) for group G.
template <int G, typename R>
__device__ __forceinline__ void run_group(const R* __restrict__ stage, const int* __restrict__ s_cs, int cb, int c0,
                                          int c1, const Piece<R>& px, const Piece<R>& py, R inv_dx, R fi, R fj,
                                          R* acc) {
    sweep_cell<G, 0>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
    sweep_cell<G, 1>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
    sweep_cell<G, 2>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
    sweep_cell<G, 3>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
}

// Write group G's column sums (deterministic: to its partial row; fast: into
// the shared tile).
template <int G, typename R, bool kDeterministic>
__device__ __forceinline__ void flush_group(const R* acc, R* acc_smem, int l, int a, int bb) {
    flush_channel<G, 0, R, kDeterministic>(acc, acc_smem, l, a, bb);
    flush_channel<G, 1, R, kDeterministic>(acc, acc_smem, l, a, bb);
    flush_channel<G, 2, R, kDeterministic>(acc, acc_smem, l, a, bb);
    flush_channel<G, 3, R, kDeterministic>(acc, acc_smem, l, a, bb);
    if (G == 1) flush_channel<1, 4, R, kDeterministic>(acc, acc_smem, l, a, bb);
}

template <typename R, bool kDeterministic>
__global__ void __launch_bounds__(kP2GThreads, sizeof(R) == 4 ? 2 : 1)
    k_p2g(const SceneDev<R>* __restrict__ sc, PState<R> st, PAux<R> aux, BinDev bin, R* __restrict__ tile,
          const Counters* __restrict__ cnt) {
    constexpr int CH = P2GChunk<R>::value;
    constexpr int NA = 6 * 5;  // accumulator words (group 1 uses all 30, group 0 the first 24)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* stage = reinterpret_cast<R*>(smem_raw);          // [CH][kRec]
    R* acc_smem = stage + (size_t)CH * kRec;             // det: [144][54] column sums; fast: [9][216] tile
    __shared__ int s_cs[65];

    const int t = threadIdx.x;
    const int group = t / kGroupThreads;
    const int l = t - group * kGroupThreads;
    const bool worker = l < kColumns;
    const int colcell = l / 9;  // (cx, cy) = (colcell >> 2, colcell & 3)
    const int col = l - colcell * 9;
    const int ci = col / 3, cj = col - (col / 3) * 3;
    const int cb = (colcell >> 2) * 16 + (colcell & 3) * 4;  // first cell (cz = 0) of the z-column
    const R inv_dx = sc->inv_dx;
    const R fi = R(ci), fj = R(cj);
    Piece<R> px, py;
    px.init(ci, inv_dx);
    py.init(cj, inv_dx);
    const int nb = min(cnt->n_blocks, bin.nb_cap);

    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        for (int q = t; q < 65; q += kP2GThreads) s_cs[q] = bin.cell_start[(int64_t)b * 64 + q];
        if (!kDeterministic)
            for (int q = t; q < kP2GChannels * kWindowNodes; q += kP2GThreads) acc_smem[q] = R(0);
        int bx, by, bz;
        page_coords(bin.block_keys[b], bx, by, bz);
        __syncthreads();
        const int bs = s_cs[0], be = s_cs[64];
        R acc[NA];
#pragma unroll
        for (int q = 0; q < NA; ++q) acc[q] = R(0);
        for (int c0 = bs; c0 < be; c0 += CH) {
            const int c1 = min(be, c0 + CH);
            for (int p = t; p < c1 - c0; p += kP2GThreads) {
                const int slot = c0 + p;
                const int o = bin.perm[slot];
                const uint32_t cell = bin.keys_sorted[slot] & 63u;
                const int base[3] = {4 * bx + (int)(cell >> 4), 4 * by + (int)((cell >> 2) & 3),
                                     4 * bz + (int)(cell & 3)};
                stage_particle(sc, st, aux, o, base, stage + (size_t)p * kRec);
            }
            __syncthreads();
            if (worker) {
                if (group == 0)
                    run_group<0>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
                else
                    run_group<1>(stage, s_cs, cb, c0, c1, px, py, inv_dx, fi, fj, acc);
            }
            __syncthreads();
        }
        R* out = tile + (int64_t)b * kP2GChannels * kWindowNodes;
        {
            const int a = (colcell >> 2) + ci, bb = (colcell & 3) + cj;
            if (worker) {
                if (group == 0)
                    flush_group<0, R, kDeterministic>(acc, acc_smem, l, a, bb);
                else
                    flush_group<1, R, kDeterministic>(acc, acc_smem, l, a, bb);
            }
        }
        __syncthreads();
        if (kDeterministic) {
            // window node (a, b, c): sum over cell columns (cx, cy) with stencil
            // column (a - cx, b - cy), in fixed order
            for (int oi = t; oi < kP2GChannels * kWindowNodes; oi += kP2GThreads) {
                const int ch = oi / kWindowNodes;
                const int node = oi - ch * kWindowNodes;
                const int a = node / 36, bb = (node / 6) % 6, c = node % 6;
                R sum = R(0);
                for (int cx = max(0, a - 2); cx <= min(3, a); ++cx)
                    for (int cy = max(0, bb - 2); cy <= min(3, bb); ++cy) {
                        const int thr = (cx * 4 + cy) * 9 + (a - cx) * 3 + (bb - cy);
                        sum += acc_smem[thr * kColAcc + c * 9 + ch];
                    }
                out[oi] = sum;
            }
        } else {
            for (int oi = t; oi < kP2GChannels * kWindowNodes; oi += kP2GThreads) out[oi] = acc_smem[oi];
        }
        __syncthreads();
    }
}

template <typename R, bool kDet>
size_t p2g_smem_bytes() {
    return sizeof(R) * ((size_t)P2GChunk<R>::value * kRec +
                        (kDet ? (size_t)kColumns * kColAcc : (size_t)kP2GChannels * kWindowNodes));
}

template <typename R>
cudaError_t prepare_p2g() {
    cudaError_t e = cudaFuncSetAttribute(k_p2g<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)p2g_smem_bytes<R, true>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_p2g<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p2g_smem_bytes<R, false>());
}
template cudaError_t prepare_p2g<float>();
template cudaError_t prepare_p2g<double>();

template <typename R>
cudaError_t launch_p2g(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const int per_sm = sizeof(R) == 4 ? 2 : 1;
    const int ctas = max(1, min(bin.nb_cap, cfg.num_sms * per_sm));
    R* tile = reinterpret_cast<R*>(grid.tile);
    if (cfg.deterministic)
        k_p2g<R, true><<<ctas, kP2GThreads, p2g_smem_bytes<R, true>(), stream>>>(sc, st, aux, bin, tile, cnt);
    else
        k_p2g<R, false><<<ctas, kP2GThreads, p2g_smem_bytes<R, false>(), stream>>>(sc, st, aux, bin, tile, cnt);
    return cudaGetLastError();
}

template cudaError_t launch_p2g<float>(const SceneDev<float>*, const PState<float>&, const PAux<float>&, BinDev,
                                       GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_p2g<double>(const SceneDev<double>*, const PState<double>&, const PAux<double>&, BinDev,
                                        GridDev, Counters*, LaunchCfg, cudaStream_t);

}  // namespace gmpm
