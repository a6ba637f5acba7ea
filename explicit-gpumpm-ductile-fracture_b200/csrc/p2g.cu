// P2G: APIC particle-to-grid transfer on SPGrid pages (P2G_APIC,
// P2GKernal.cu:512-702) plus the phase-field channels (volP2G_APIC,
// preConditionP2G_APIC, AxP2G_APIC: P2GKernal.cu:897-1326).
//
// Each CTA walks its particle pages (grid-stride) in chunks of up to
// P2GChunk sorted slots (a whole page of 8 particles per cell in FP32).  A
// page's particles share the page's 6x6x6 node window and, within a cell,
// the same 3x3x3 stencil.  Between substeps the particle planes are in the
// previous sorted order and perm is close to the identity, so the 28 raw
// input planes of the next chunk are fetched as contiguous windows of
// previous slots with bulk copies (one thread issues them; the tensor memory
// accelerator moves the data) while the current chunk is swept.  Particles
// whose previous slot falls outside the window (they changed page) are read
// directly.  Each thread then turns one particle's raw words into a 44-word
// record.
//
// Work split: one warp per cell z-column (cx, cy) of the page; lane
// (g, i, j) = channel group g (0..2) x stencil column (i, j).  A warp sweeps
// its column's cells (cx, cy, 0..3) in order, all lanes on the same particle,
// so control flow is uniform.  Lane (g, i, j) owns window nodes
// (cx+i, cy+j, 0..5) for its group's three channels:
//   g = 0: momentum x, mass, damage weight
//   g = 1: momentum y, weight, V w
//   g = 2: momentum z, V w FP, grad w . q (phase-field flux)
// Every particle of cell cz adds to nodes cz..cz+2 with register indices
// fixed at compile time (the sweep over cz is unrolled), so the sums stay in
// registers: no shuffles and no per-particle atomics.
//
// Deterministic mode: after a page's last chunk the column sums are gathered
// per window node in a fixed order (at most 9 terms, compensated) and written once to the
// page's tile in HBM, so results are bitwise reproducible.  Fast mode:
// columns add into a shared tile with atomics.  The grid kernel sums the
// eight page tiles overlapping each grid page in fixed slot order either way.
#include <cstdint>

#include "async_copy.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace gmpm {

constexpr int kP2GWarps = 16;  // one per cell z-column (cx, cy)
constexpr int kP2GThreads = 32 * kP2GWarps;
constexpr int kColumns = 144;  // 16 cell z-columns x 9 stencil columns
// Page flush: column sums channel-major, [channel][stencil column (144)][z (6)], the channel stride padded
// so that the three channel groups of a warp's stores fall in different banks.  A gather step of one
// channel over consecutive window nodes then reads consecutive words.
constexpr int kFlushChStride = kColumns * 6 + 8;
constexpr int kRec = 44;       // words per staged particle record

template <typename R> struct P2GChunk;
template <> struct P2GChunk<float> { static constexpr int value = 512; };
template <> struct P2GChunk<double> { static constexpr int value = 256; };

// Record layout: 8 common words (the x and y offsets from the base node in
// cells, xp/dx; the three z weights and their gradients), then one 12-word
// block per channel group g at RF_BLOCK + 12 g:
//   U, A0, A1, A2 | S0, S1, S2, s1 | t0, t1, t2, t3
// with, for a lane of stencil column (i, j) and node k of the sweep,
//   momentum_g += w (U + A0 i + A1 j + A2 k) + (S0 gxy0 + S1 gxy1) wz + S2 wxy gz
//   second     += s1 w
//   third      += (t0 wxy + t1 gxy0 + t2 gxy1) wz + t3 wxy gz
// where U = m v_g - (m B D^-1 xp)_g, A = dx (m B D^-1) row g, S = -dt V0 P F^T
// row g.  s1 = (m, 1, V FP); t = (c,0,0,0), (V,0,0,0), (0, q0, q1, q2).
enum RecField : int { RF_XP0 = 0, RF_XP1 = 1, RF_WZ = 2, RF_GZ = 5, RF_BLOCK = 8 };
static_assert(RF_BLOCK + 3 * 12 == kRec, "record layout");

// Raw particle planes, in staging order.
enum RawField : int {
    RW_X = 0, RW_V = 3, RW_B = 6, RW_SIG = 15, RW_C = 21, RW_M = 22, RW_VOL = 23, RW_FP = 24, RW_Q = 25,
    kRawWords = 28
};

// Staging window of previous slots: the chunk's CH slots plus kMargin on
// either side; planes padded in shared memory to spread banks.
constexpr int kMargin = 64;
template <typename R>
struct Staging {
    static constexpr int CH = P2GChunk<R>::value;
    static constexpr int W = CH + 2 * kMargin;             // window length (elements)
    static constexpr int WS = W + (int)(16 / sizeof(R));   // plane stride in shared memory
    static_assert(W <= kPlanePad, "window fits the plane padding");
    static_assert((W * sizeof(R)) % 16 == 0 && (WS * sizeof(R)) % 16 == 0, "bulk copy granularity");
};

// Device pointer of raw plane q.
template <typename R>
__device__ __forceinline__ const R* raw_plane(const PState<R>& st, const PAux<R>& aux, int q) {
    if (q < RW_V) return st.x[q - RW_X];
    if (q < RW_B) return aux.v[q - RW_V];
    if (q < RW_SIG) return aux.B[q - RW_B];
    if (q < RW_C) return aux.sigma[q - RW_SIG];
    if (q == RW_C) return st.c;
    if (q == RW_M) return st.m;
    if (q == RW_VOL) return aux.vol;
    if (q == RW_FP) return aux.FP;
    return aux.q[q - RW_Q];
}

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

// Build the particle's record from its raw words.
template <typename R>
__device__ __forceinline__ void build_record(const SceneDev<R>* __restrict__ sc, const int base[3], const R* raw,
                                             R* rec) {
    const R dx = sc->dx, inv_dx = sc->inv_dx, dt = sc->dt, Dinv = sc->Dinv;
    R xp[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xp[a] = raw[RW_X + a] - R(base[a]) * dx;
    R out[kRec];
    // x and y offsets in cells: the product every lane's weight needs, formed once
    out[RF_XP0] = xp[0] * inv_dx;
    out[RF_XP1] = xp[1] * inv_dx;
    bspline1d(xp[2], inv_dx, out + RF_WZ, out + RF_GZ);
    const R m = raw[RW_M];
    const R V = raw[RW_VOL];
    R mB[9];  // m B D^-1, (r,c) at 3r+c; B planes are column-major (r + 3c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) mB[3 * r + c] = m * raw[RW_B + r + 3 * c] * Dinv;
    // -dt sigma, sigma stored xx yy zz xy xz yz
    R S[9];
    S[0] = -dt * raw[RW_SIG + 0];
    S[4] = -dt * raw[RW_SIG + 1];
    S[8] = -dt * raw[RW_SIG + 2];
    S[1] = S[3] = -dt * raw[RW_SIG + 3];
    S[2] = S[6] = -dt * raw[RW_SIG + 4];
    S[5] = S[7] = -dt * raw[RW_SIG + 5];
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        R* blk = out + RF_BLOCK + 12 * g;
        blk[0] = m * raw[RW_V + g] - (mB[3 * g] * xp[0] + mB[3 * g + 1] * xp[1] + mB[3 * g + 2] * xp[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            blk[1 + c] = dx * mB[3 * g + c];
            blk[4 + c] = S[3 * g + c];
        }
    }
    R* b0 = out + RF_BLOCK;
    R* b1 = b0 + 12;
    R* b2 = b1 + 12;
    b0[7] = m;
    b0[8] = raw[RW_C];
    b0[9] = b0[10] = b0[11] = R(0);
    b1[7] = R(1);
    b1[8] = V;
    b1[9] = b1[10] = b1[11] = R(0);
    b2[7] = V * raw[RW_FP];
    b2[8] = R(0);
    b2[9] = raw[RW_Q + 0];
    b2[10] = raw[RW_Q + 1];
    b2[11] = raw[RW_Q + 2];
    static_assert((kRec * sizeof(R)) % 16 == 0, "record must be whole 16-byte words");
#pragma unroll
    for (int q = 0; q < (int)(kRec * sizeof(R) / 16); ++q)
        reinterpret_cast<uint4*>(rec)[q] = reinterpret_cast<const uint4*>(out)[q];
}

// Per-lane constants of the B-spline piece of stencil node i along one axis,
// written around z = xp/dx - shift: w = a z^2 + b, dw/dx = c z.
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

template <int NW, typename R>
__device__ __forceinline__ void load_words(const R* __restrict__ src, R* dst) {
    static_assert((NW * sizeof(R)) % 16 == 0, "whole 16-byte words");
#pragma unroll
    for (int q = 0; q < (int)(NW * sizeof(R) / 16); ++q)
        reinterpret_cast<uint4*>(dst)[q] = reinterpret_cast<const uint4*>(src)[q];
}

// One particle of cell z-index CZ into a lane's 6 z-nodes x 3 channels.
template <int CZ, typename R>
__device__ __forceinline__ void accumulate(const R* __restrict__ rec, int g, const Piece<R>& px, const Piece<R>& py,
                                           R fi, R fj, R* acc) {
    R cw[8], bw[12];
    load_words<8>(rec, cw);
    load_words<12>(rec + RF_BLOCK + 12 * g, bw);
    R wx, gx, wy, gy;
    px.eval(cw[RF_XP0], wx, gx);
    py.eval(cw[RF_XP1], wy, gy);
    const R wxy = wx * wy, gxy0 = gx * wy, gxy1 = wx * gy;
    const R al = bw[4] * gxy0 + bw[5] * gxy1, be = bw[6] * wxy;
    const R s1w = bw[7] * wxy;
    const R gam = bw[8] * wxy + bw[9] * gxy0 + bw[10] * gxy1, del = bw[11] * wxy;
    // momentum at node k: wz (wxy u_k + al) + gz be with u_k = u0 + k A2, i.e.
    // wz (alpha + k beta) + gz be
    const R u0 = bw[0] + bw[1] * fi + bw[2] * fj;
    const R alpha = wxy * u0 + al, beta = wxy * bw[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R wz = cw[RF_WZ + k], gz = cw[RF_GZ + k];
        const R tk = k == 0 ? alpha : (k == 1 ? alpha + beta : alpha + R(2) * beta);
        R* A = acc + 3 * (CZ + k);
        A[0] += wz * tk + be * gz;
        A[1] += s1w * wz;
        A[2] += gam * wz + del * gz;
    }
}

template <int CZ, typename R>
__device__ __forceinline__ void sweep_cell(const R* __restrict__ recs, const int* __restrict__ s_cs, int cb, int c0,
                                           int c1, int g, const Piece<R>& px, const Piece<R>& py, R fi, R fj,
                                           R* acc) {
    const int lo = max(s_cs[cb + CZ], c0) - c0, hi = min(s_cs[cb + CZ + 1], c1) - c0;
#pragma unroll 4
    for (int p = lo; p < hi; ++p) accumulate<CZ>(recs + (size_t)p * kRec, g, px, py, fi, fj, acc);
}

// Channel of slot q (0..2) of group g's accumulator row.
__device__ __forceinline__ int group_channel(int g, int q) {
    if (q == 0) return CH_P0 + g;
    if (q == 1) return g == 0 ? CH_M : (g == 1 ? CH_W : CH_VWFP);
    return g == 0 ? CH_CW : (g == 1 ? CH_VW : CH_KC);
}

// Chunk sequence of one CTA: its pages b + k g (b, g: the CTA's index and the
// CTA count of its scene's share of the launch), each cut into runs of CH
// slots.  Every thread runs the same iterator.
template <int CH>
struct ChunkIter {
    int page, next, end;  // current page, next run start, page end
    int nbs, nbe;         // slot range of the following page (loaded one page ahead)
    int stride;           // CTAs of the scene's share of the launch
    __device__ void init(const BinDev& bin, int nb, VB vb) {
        page = vb.b;
        stride = vb.g;
        next = end = 0;
        if (page < nb) {
            next = bin.cell_start[(int64_t)page * 64];
            end = bin.cell_start[(int64_t)page * 64 + 64];
        }
        preload(bin, nb);
    }
    __device__ void preload(const BinDev& bin, int nb) {
        const int q = page + stride;
        nbs = nbe = 0;
        if (q < nb) {
            nbs = bin.cell_start[(int64_t)q * 64];
            nbe = bin.cell_start[(int64_t)q * 64 + 64];
        }
    }
    // Next chunk (page, first slot, count, last chunk of its page); count 0 when done.
    __device__ void step(const BinDev& bin, int nb, int& b, int& s0, int& n, int& last) {
        while (page < nb && next >= end) {
            page += stride;
            next = nbs;
            end = nbe;
            if (page < nb) preload(bin, nb);
        }
        if (page < nb) {
            b = page;
            s0 = next;
            n = min(CH, end - next);
            next += CH;
            last = next >= end;
        } else {
            b = -1;
            s0 = n = last = 0;
        }
    }
};

template <int CH>
struct P2GMeta {
    int32_t o[3][CH];     // previous slot per chunk slot; 3 buffers
    uint32_t key[3][CH];  // sorted key per chunk slot
    int32_t cs[3][68];    // cell starts of the chunk's page (65 used)
    uint32_t bkey[3];
    int32_t chunk[3][4];  // page, first slot, count (0: none), last chunk of page
    int64_t win[3];       // first previous slot of the chunk's staging window
    uint64_t bar;         // completion of the staging bulk copies
    int abort;            // a bounded wait gave up
    // page flush: the column-sum offsets of window node n's terms, in summing order
    // (cell column cx then cy ascending), and their count
    uint16_t goff[kWindowNodes][9];
    uint8_t gcnt[kWindowNodes];
};

// Start of the staging window of a chunk: the median over three particles of
// (previous slot - slot) estimates the chunk's shift between the orders.
template <typename R, int CH>
__device__ __forceinline__ int64_t window_start(const int32_t* o, int n, int64_t stride) {
    const int64_t d0 = o[0], d1 = (int64_t)o[n / 2] - n / 2, d2 = (int64_t)o[n - 1] - (n - 1);
    const int64_t med = max(min(d0, d1), min(max(d0, d1), d2));
    int64_t w = (med - kMargin) & ~(int64_t)3;
    w = min(w, stride - Staging<R>::W);
    return max(w, (int64_t)0);
}

// Thread 0: bulk copies of the 28 raw planes over the chunk's window.
template <typename R, int CH>
__device__ __forceinline__ void issue_staging(P2GMeta<CH>& S, R* stage, int64_t w0, const PState<R>& st,
                                              const PAux<R>& aux) {
    constexpr int W = Staging<R>::W, WS = Staging<R>::WS;
    fence_proxy_async_shared();
    mbar_arrive_expect_tx(&S.bar, (unsigned)(kRawWords * W * sizeof(R)));
#pragma unroll
    for (int q = 0; q < kRawWords; ++q)
        bulk_copy_g2s(stage + (size_t)q * WS, raw_plane(st, aux, q) + w0, (unsigned)(W * sizeof(R)), &S.bar);
}

template <int CH>
__device__ __forceinline__ void issue_p2g_meta(P2GMeta<CH>& S, int m, int b, int s0, int n, const BinDev& bin) {
    const int t = threadIdx.x;
    if (n <= 0) return;
    for (int p = t; p < n; p += kP2GThreads) {
        cp_async_elem(&S.o[m][p], &bin.perm[s0 + p]);
        cp_async_elem(&S.key[m][p], &bin.keys_sorted[s0 + p]);
    }
    if (t < 65) cp_async_elem(&S.cs[m][t], &bin.cell_start[(int64_t)b * 64 + t]);
    if (t == 65) cp_async_elem(&S.bkey[m], &bin.block_keys[b]);
}

template <typename R>
constexpr size_t p2g_rec_bytes() {
    return sizeof(R) * (size_t)P2GChunk<R>::value * kRec;
}
template <typename R>
constexpr size_t p2g_stage_bytes() {
    return sizeof(R) * (size_t)kRawWords * Staging<R>::WS;
}

template <typename R, bool kDeterministic>
__device__ __forceinline__ void p2g_body(VB vb, const SceneDev<R>* __restrict__ sc, const PState<R>& st,
                                         const PAux<R>& aux, const BinDev& bin, R* __restrict__ tile,
                                         Counters* __restrict__ cnt) {
    constexpr int CH = P2GChunk<R>::value;
    constexpr int W = Staging<R>::W, WS = Staging<R>::WS;
    static_assert(sizeof(R) * kP2GChannels * kFlushChStride <= p2g_rec_bytes<R>(), "column sums fit the record buffer");
    static_assert(sizeof(R) * kP2GChannels * kWindowNodes <= p2g_rec_bytes<R>(), "tile fits the record buffer");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* recs = reinterpret_cast<R*>(smem_raw);                          // [CH][kRec] particle records
    R* stage = reinterpret_cast<R*>(smem_raw + p2g_rec_bytes<R>());   // [kRawWords][WS] raw planes
    P2GMeta<CH>& S = *reinterpret_cast<P2GMeta<CH>*>(smem_raw + p2g_rec_bytes<R>() + p2g_stage_bytes<R>());

    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const int le = lane < 27 ? lane : lane - 27;  // lanes 27..31 shadow lanes 0..4 and never flush
    const int g = le / 9;
    const int col = le - g * 9;
    const int ci = col / 3, cj = col - ci * 3;
    // Warp w owns z-column (cx, cy) = (w / 4, (w - cx) mod 4): the four warps
    // of a scheduler (w mod 4) then hold one column of every cx and every cy,
    // so a page's empty rows or slabs of cells do not all land on one scheduler.
    const int wcx = warp >> 2, wcy = ((warp & 3) - wcx) & 3;
    const int cb = wcx * 16 + wcy * 4;  // first cell (cz = 0) of the z-column
    const R inv_dx = sc->inv_dx;
    const R fi = R(ci), fj = R(cj);
    Piece<R> px, py;
    px.init(ci, inv_dx);
    py.init(cj, inv_dx);
    const int nb = min(cnt->n_blocks, bin.nb_cap);

    // prologue: meta of chunks 0 and 1, staging of chunk 0
    ChunkIter<CH> it;
    it.init(bin, nb, vb);
    {
        int b0, s0, n0, l0, b1, s1, n1, l1;
        it.step(bin, nb, b0, s0, n0, l0);
        it.step(bin, nb, b1, s1, n1, l1);
        if (t < kWindowNodes) {
            const int na = t / 36, nbb = (t / 6) % 6, nc = t % 6;
            int q = 0;
            for (int cx = max(0, na - 2); cx <= min(3, na); ++cx)
                for (int cy = max(0, nbb - 2); cy <= min(3, nbb); ++cy)
                    S.goff[t][q++] = (uint16_t)(((cx * 4 + cy) * 9 + (na - cx) * 3 + (nbb - cy)) * 6 + nc);
            S.gcnt[t] = (uint8_t)q;
        }
        if (t == 0) {
            S.chunk[0][0] = b0; S.chunk[0][1] = s0; S.chunk[0][2] = n0; S.chunk[0][3] = l0;
            S.chunk[1][0] = b1; S.chunk[1][1] = s1; S.chunk[1][2] = n1; S.chunk[1][3] = l1;
            S.abort = 0;
            mbar_init(&S.bar, 1);
            mbar_init_fence();
        }
        issue_p2g_meta(S, 0, b0, s0, n0, bin);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        if (t == 0 && n0 > 0) {
            S.win[0] = window_start<R, CH>(S.o[0], n0, st.stride);
            issue_staging(S, stage, S.win[0], st, aux);
        }
        issue_p2g_meta(S, 1, b1, s1, n1, bin);
        cp_async_commit();
    }

    R acc[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) acc[q] = R(0);

    for (int k = 0;; ++k) {
        const int m0 = k % 3, m1 = (k + 1) % 3, m2 = (k + 2) % 3;
        cp_async_wait_all();
        const int n0 = S.chunk[m0][2];
        if (n0 > 0 && !mbar_wait(&S.bar, (unsigned)(k & 1))) S.abort = 1;
        __syncthreads();
        if (n0 <= 0 || S.abort) break;
        const int b0 = S.chunk[m0][0], c0 = S.chunk[m0][1], last0 = S.chunk[m0][3];
        // records of chunk k from the staged window (or directly for particles outside it)
        {
            int bx, by, bz;
            page_coords(S.bkey[m0], bx, by, bz);
            const int64_t w0 = S.win[m0];
            for (int p = t; p < n0; p += kP2GThreads) {
                const int o = S.o[m0][p];
                const int64_t r = (int64_t)o - w0;
                R raw[kRawWords];
                if (r >= 0 && r < W) {
#pragma unroll
                    for (int q = 0; q < kRawWords; ++q) raw[q] = stage[(size_t)q * WS + r];
                } else {
#pragma unroll
                    for (int q = 0; q < kRawWords; ++q) raw[q] = raw_plane(st, aux, q)[o];
                }
                const uint32_t cell = S.key[m0][p] & 63u;
                const int base[3] = {4 * bx + (int)(cell >> 4), 4 * by + (int)((cell >> 2) & 3),
                                     4 * bz + (int)(cell & 3)};
                build_record(sc, base, raw, recs + (size_t)p * kRec);
            }
        }
        __syncthreads();
        {
            // chunk k+1: staging (the buffer is free now); chunk k+2: iterator step, descriptor and meta.
            // The staging copies are issued by the warp whose column holds the fewest of this chunk's
            // particles, so that the issue delays the sweep least (each warp finds it the same way).
            const int n1 = S.chunk[m1][2];
            int issuer;
            {
                const int* cs = S.cs[m0];
                const int c1 = c0 + n0;
                const int lw = lane & 15;
                const int lcx = lw >> 2, lcy = ((lw & 3) - lcx) & 3, lcb = lcx * 16 + lcy * 4;
                int key = ((min(max(cs[lcb + 4], c0), c1) - min(max(cs[lcb], c0), c1)) << 4) | lw;
#pragma unroll
                for (int off = 8; off > 0; off >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, off));
                issuer = key & 15;
            }
            if (warp == issuer && lane == 0 && n1 > 0) {
                S.win[m1] = window_start<R, CH>(S.o[m1], n1, st.stride);
                issue_staging(S, stage, S.win[m1], st, aux);
            }
            int b2, s2, n2, l2;
            it.step(bin, nb, b2, s2, n2, l2);
            if (t == 0) {
                S.chunk[m2][0] = b2;
                S.chunk[m2][1] = s2;
                S.chunk[m2][2] = n2;
                S.chunk[m2][3] = l2;
            }
            issue_p2g_meta(S, m2, b2, s2, n2, bin);
            cp_async_commit();
        }
        {
            const int* s_cs = S.cs[m0];
            const int c1 = c0 + n0;
            sweep_cell<0>(recs, s_cs, cb, c0, c1, g, px, py, fi, fj, acc);
            sweep_cell<1>(recs, s_cs, cb, c0, c1, g, px, py, fi, fj, acc);
            sweep_cell<2>(recs, s_cs, cb, c0, c1, g, px, py, fi, fj, acc);
            sweep_cell<3>(recs, s_cs, cb, c0, c1, g, px, py, fi, fj, acc);
        }
        if (!last0) continue;

        // Page done: column sums -> the page's tile.  The sums go to the
        // record buffer, which is free once every warp is past its sweep.
        __syncthreads();
        R* acc_smem = recs;
        const int a = wcx + ci, bb = wcy + cj;
        if (!kDeterministic) {
            for (int q = t; q < kP2GChannels * kWindowNodes; q += kP2GThreads) acc_smem[q] = R(0);
            __syncthreads();
        }
        if (lane < 27) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int ch = group_channel(g, q);
#pragma unroll
                for (int z = 0; z < 6; ++z) {
                    if (kDeterministic)
                        acc_smem[ch * kFlushChStride + ((wcx * 4 + wcy) * 9 + col) * 6 + z] = acc[3 * z + q];
                    else
                        atomicAdd(&acc_smem[ch * kWindowNodes + a * 36 + bb * 6 + z], acc[3 * z + q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 18; ++q) acc[q] = R(0);
        __syncthreads();
        R* out = tile + (int64_t)b0 * kP2GChannels * kWindowNodes;
        if (kDeterministic) {
            // tile value (ch, n): window node n = (a, b, c) sums cell columns (cx, cy) with stencil
            // column (a - cx, b - cy), cx then cy ascending (compensated).  One (channel, node) sum per
            // thread step over all threads: the sums are short dependent chains, so spreading them keeps
            // every warp busy where one thread per node left most of the CTA waiting.
            constexpr int kItems = (kP2GChannels * kWindowNodes + kP2GThreads - 1) / kP2GThreads;
            int base[kItems], cnt[kItems];
            R sum[kItems], comp[kItems];
#pragma unroll
            for (int i = 0; i < kItems; ++i) {
                const int w = t + i * kP2GThreads;
                const int ch = w / kWindowNodes;
                const int n = w - ch * kWindowNodes;
                const bool ok = w < kP2GChannels * kWindowNodes;
                base[i] = ok ? n * 9 : 0;
                cnt[i] = ok ? S.gcnt[n] : 0;
                sum[i] = comp[i] = R(0);
                base[i] = (base[i] << 4) | ch;  // node's offset row and channel
            }
#pragma unroll
            for (int q = 0; q < 9; ++q)
#pragma unroll
                for (int i = 0; i < kItems; ++i)
                    if (q < cnt[i])
                        kahan_add(sum[i], comp[i],
                                  acc_smem[(base[i] & 15) * kFlushChStride + (&S.goff[0][0])[(base[i] >> 4) + q]]);
#pragma unroll
            for (int i = 0; i < kItems; ++i) {
                const int w = t + i * kP2GThreads;
                if (w < kP2GChannels * kWindowNodes) out[w] = sum[i];
            }
        } else {
            for (int oi = t; oi < kP2GChannels * kWindowNodes; oi += kP2GThreads) out[oi] = acc_smem[oi];
        }
        // The record buffer is rebuilt only after the next loop-top barrier.
    }
    cp_async_wait_all();
    if (S.abort) {
        // A staging copy may still be in flight: wait for it (bounded) before
        // the CTA's shared memory goes away, and report.
        if (t == 0) {
            raise_flag(cnt, GMPM_FLAG_COPY_TIMEOUT);
            mbar_wait(&S.bar, 0u);
            mbar_wait(&S.bar, 1u);
        }
    }
}

template <typename R, bool kDeterministic>
__global__ void __launch_bounds__(kP2GThreads, 1)
    k_p2g(const SceneDev<R>* __restrict__ sc, PState<R> st, PAux<R> aux, BinDev bin, R* __restrict__ tile,
          Counters* __restrict__ cnt) {
    p2g_body<R, kDeterministic>(own_blocks(), sc, st, aux, bin, tile, cnt);
}

// Batched launch: the same body for the scene that owns this CTA.
template <typename R, bool kDeterministic>
__global__ void __launch_bounds__(kP2GThreads, 1)
    k_batch_p2g(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    p2g_body<R, kDeterministic>(vb, a.sc, a.in, a.aux, a.bin, reinterpret_cast<R*>(a.grid.tile), a.cnt);
}

template <typename R>
size_t p2g_smem_bytes() {
    return p2g_rec_bytes<R>() + p2g_stage_bytes<R>() + sizeof(P2GMeta<P2GChunk<R>::value>);
}

template <typename R>
cudaError_t prepare_p2g() {
    const int smem = (int)p2g_smem_bytes<R>();
    cudaError_t e = cudaFuncSetAttribute(k_p2g<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_p2g<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_p2g<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_p2g<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

template <typename R>
cudaError_t launch_batch_p2g(const SceneArgs<R>* A, const BatchPlan& P, cudaStream_t s) {
    const dim3 grid((unsigned)P.total[BM_P2G]);
    if (P.deterministic)
        return launch_kernel(k_batch_p2g<R, true>, grid, dim3(kP2GThreads), p2g_smem_bytes<R>(), s, A, P.start[BM_P2G],
                             P.n_scenes);
    return launch_kernel(k_batch_p2g<R, false>, grid, dim3(kP2GThreads), p2g_smem_bytes<R>(), s, A, P.start[BM_P2G],
                         P.n_scenes);
}
template cudaError_t launch_batch_p2g<float>(const SceneArgs<float>*, const BatchPlan&, cudaStream_t);
template cudaError_t launch_batch_p2g<double>(const SceneArgs<double>*, const BatchPlan&, cudaStream_t);
template cudaError_t prepare_p2g<float>();
template cudaError_t prepare_p2g<double>();

template <typename R>
cudaError_t launch_p2g(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const int ctas = max(1, min(bin.nb_cap, cfg.num_sms));
    R* tile = reinterpret_cast<R*>(grid.tile);
    if (cfg.deterministic)
        k_p2g<R, true><<<ctas, kP2GThreads, p2g_smem_bytes<R>(), stream>>>(sc, st, aux, bin, tile, cnt);
    else
        k_p2g<R, false><<<ctas, kP2GThreads, p2g_smem_bytes<R>(), stream>>>(sc, st, aux, bin, tile, cnt);
    return cudaGetLastError();
}

template cudaError_t launch_p2g<float>(const SceneDev<float>*, const PState<float>&, const PAux<float>&, BinDev,
                                       GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_p2g<double>(const SceneDev<double>*, const PState<double>&, const PAux<double>&, BinDev,
                                        GridDev, Counters*, LaunchCfg, cudaStream_t);

}  // namespace gmpm
